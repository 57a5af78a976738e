// GPU-resident IR producer: the left / right impulse responses of a shoebox room
// written straight into device memory, for tanb_convolution_update_response_td_device
// (the GPU path of TrueAudioVR::generateRoomResponse with GENROOM_USE_GPU_MEM,
// samples/src/TrueAudioVR/TrueAudioVR.cpp:659-786; kernels
// Kernels/GenerateRoomResponse.cl:206-321 and Kernels/Fill.cl).
//
// Per ear, one thread per image source (index i_x in [-n_W, n_W] along the
// width, etc., over the grid the reference launches: local size 4, so the
// last index exists only when 2 n_W is not a multiple of 4). An image at
// distance d lands at sample 1 + (int)(d / 340 * rate) with gain
// damp^walls x distance gain; early images (before the HRTF cutoff) add the
// head filter lowPass + hf * highPass (hf from the angle to the ear vector),
// late ones a single tap. Each contribution is truncated to a 2^-26 fixed
// point value, as the reference, and summed with 64-bit integer atomics, so
// the sum is exact and independent of thread order; a second kernel converts
// to float and clears the accumulator. Differences from the reference: damp^k
// by repeated multiplication (native_powr is implementation-defined), sqrt
// correctly rounded, 64-bit sums converted as signed (the reference's int32
// sums can wrap and Fill.cl converts them as unsigned). Every product and sum
// is an explicit round-to-nearest operation, so the results are reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/tanb.h"
#include "tanb_internal.h"

namespace tanb {
namespace {

struct RoomEar {
  float W, H, L;
  float dLeft, dRight, dTop, dBottom, dFront, dBack;
  float sx, sy, sz;
  float hx, hy, hz;
  float evx, evy, evz, earV;
  float maxGain, dMin;
  int rate, length, hrtfLength, filterLength;
  int numRefX, numRefY, numRefZ;  // 2 n per axis
  int cx, cy, cz;                 // grid extent per axis (indices 0 .. c-1)
  float lp[64], hp[64];
};

__device__ __forceinline__ float pow_int(float b, int k) {
  float r = 1.0f;
  for (int i = 0; i < k; ++i) r = __fmul_rn(r, b);
  return r;
}

__device__ __forceinline__ float image_pos(int idx, float size, float s) {
  const float a = (idx % 2 == 0) ? (float)idx : (float)(idx + 1);
  const float b = (idx % 2 == 0) ? 1.0f : -1.0f;
  return __fadd_rn(__fmul_rn(a, size), __fmul_rn(b, s));
}

__global__ void room_images_kernel(RoomEar a, unsigned long long* __restrict__ acc, long long images) {
  const float kF2I = 67108864.0f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < images;
       t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % a.cx);
    const int y = (int)((t / a.cx) % a.cy);
    const int z = (int)(t / ((long long)a.cx * a.cy));
    const int ix = x - a.numRefX / 2, iy = y - a.numRefY / 2, iz = z - a.numRefZ / 2;
    const float rx = image_pos(ix, a.W, a.sx), ry = image_pos(iy, a.H, a.sy), rz = image_pos(iz, a.L, a.sz);
    // reflections off each wall (GenerateRoomResponse.cl:261-276)
    const int kxl = ix > 0 ? ix / 2 : abs(ix - 1) / 2, kyb = iy > 0 ? iy / 2 : abs(iy - 1) / 2,
              kzb = iz > 0 ? iz / 2 : abs(iz - 1) / 2;
    const int kxr = ix > 0 ? (ix + 1) / 2 : abs(ix) / 2, kyt = iy > 0 ? (iy + 1) / 2 : abs(iy) / 2,
              kzf = iz > 0 ? (iz + 1) / 2 : abs(iz) / 2;
    float amp = pow_int(a.dRight, kxr);
    amp = __fmul_rn(amp, pow_int(a.dLeft, kxl));
    amp = __fmul_rn(amp, pow_int(a.dTop, kyt));
    amp = __fmul_rn(amp, pow_int(a.dBottom, kyb));
    amp = __fmul_rn(amp, pow_int(a.dFront, kzf));
    amp = __fmul_rn(amp, pow_int(a.dBack, kzb));
    const float dx = __fsub_rn(rx, a.hx), dy = __fsub_rn(ry, a.hy), dz = __fsub_rn(rz, a.hz);
    const float d = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
    const int fi = 1 + __float2int_rz(__fmul_rn(__fdiv_rn(d, 340.0f), (float)a.rate));
    if (fi >= a.length) continue;
    const float dr = (d <= a.dMin) ? a.maxGain : __fdiv_rn(__fmul_rn(a.maxGain, a.dMin), d);
    const float g = __fmul_rn(__fmul_rn(kF2I, amp), dr);
    if (fi < a.hrtfLength) {
      const float dp = __fadd_rn(__fadd_rn(__fmul_rn(a.evx, dx), __fmul_rn(a.evy, dy)), __fmul_rn(a.evz, dz));
      const float cosA = __fdiv_rn(dp, __fmul_rn(a.earV, d));
      const float hf = __fdiv_rn(__fadd_rn(cosA, 1.0f), 2.0f);
      const int len = min(a.filterLength, a.length - fi);
      for (int i = 0; i < len; ++i) {
        const int v = __float2int_rz(__fmul_rn(g, __fadd_rn(a.lp[i], __fmul_rn(hf, a.hp[i]))));
        atomicAdd(acc + fi + i, (unsigned long long)(long long)v);
      }
    } else {
      atomicAdd(acc + fi, (unsigned long long)(long long)__float2int_rz(g));
    }
  }
}

__global__ void room_fill_kernel(unsigned long long* __restrict__ acc, float* __restrict__ out, int length) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < length; i += gridDim.x * blockDim.x) {
    out[i] = __fdiv_rn(__ll2float_rn((long long)acc[i]), 67108864.0f);
    acc[i] = 0ull;
  }
}

int32_t rfail(int32_t code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}

}  // namespace
}  // namespace tanb

struct tanb_room_generator {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  cudaStream_t stream = nullptr;
  int max_length = 0;
  unsigned long long* acc = nullptr;  // [2][max_length], zero between calls
  cudaEvent_t done = nullptr;         // end of the last call, on whichever stream it ran
  long long images_last = 0;
};

extern "C" {

int32_t tanb_room_generator_create(tanb_context* ctx, int32_t max_length, tanb_room_generator** out) {
  if (!ctx || !out) return tanb::rfail(TANB_INVALID_POINTER, "null argument");
  *out = nullptr;
  if (max_length <= 0) return tanb::rfail(TANB_INVALID_ARG, "max_length must be > 0");
  tanb_room_generator* g = new tanb_room_generator();
  g->ctx = ctx;
  g->max_length = max_length;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&g->acc, 2 * (size_t)max_length * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(g->acc, 0, 2 * (size_t)max_length * sizeof(unsigned long long), g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    if (g->acc) cudaFree(g->acc);
    if (g->done) cudaEventDestroy(g->done);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    cudaGetLastError();
    return tanb::rfail(e == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "room generator: %s",
                       cudaGetErrorString(e));
  }
  *out = g;
  return TANB_OK;
}

int32_t tanb_room_generator_release(tanb_room_generator* g) {
  if (!g) return TANB_OK;
  {
    std::lock_guard<std::mutex> lock(g->mu);
    cudaSetDevice(g->ctx->device);
    cudaEventSynchronize(g->done);
    cudaStreamSynchronize(g->stream);
    cudaFree(g->acc);
    cudaEventDestroy(g->done);
    cudaStreamDestroy(g->stream);
  }
  delete g;
  return TANB_OK;
}

int32_t tanb_room_response(tanb_room_generator* g, const tanb_room* room, const tanb_source* source,
                           const tanb_listener* ears, int32_t sample_rate, int32_t length, float* left, float* right,
                           uint32_t flags, int32_t max_bounces, void* stream) {
  if (!g || !room || !source || !ears || !left || !right) return tanb::rfail(TANB_INVALID_POINTER, "null argument");
  if (length <= 0 || length > g->max_length)
    return tanb::rfail(TANB_INVALID_ARG, "length %d not in [1, %d]", length, g->max_length);
  if (sample_rate <= 0) return tanb::rfail(TANB_INVALID_ARG, "sample_rate must be > 0");
  if (ears->filter_length < 0 || ears->filter_length > 64)
    return tanb::rfail(TANB_INVALID_ARG, "filter_length must be in [0, 64]");
  if ((flags & TANB_GENROOM_LIMIT_BOUNCES) && max_bounces <= 0)
    return tanb::rfail(TANB_INVALID_ARG, "max_bounces must be > 0 with TANB_GENROOM_LIMIT_BOUNCES");
  std::lock_guard<std::mutex> lock(g->mu);
  cudaError_t e = cudaSetDevice(g->ctx->device);
  if (e != cudaSuccess) return tanb::rfail(TANB_FAIL, "%s", cudaGetErrorString(e));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->stream;

  // host setup, TrueAudioVR.cpp:663-731
  tanb::RoomEar a{};
  a.W = room->width;
  a.H = room->height;
  a.L = room->length;
  a.dLeft = room->damp_left;
  a.dRight = room->damp_right;
  a.dTop = room->damp_top;
  a.dBottom = room->damp_bottom;
  a.dFront = room->damp_front;
  a.dBack = room->damp_back;
  a.sx = std::min(std::max(source->x, 0.0f), a.W);
  a.sy = std::min(std::max(source->y, 0.0f), a.H);
  a.sz = std::min(std::max(source->z, 0.0f), a.L);
  const float es = ears->ear_spacing;
  float ev[4][3] = {{es / 2, 0.0f, 0.0f}, {-es / 2, 0.0f, 0.0f}, {es / 2, 0.0f, -(es / 2)}, {-es / 2, 0.0f, -es / 2}};
  const float pi = (float)3.141592653589793;
  const float sY = std::sin(ears->yaw * pi / 180), cY = std::cos(ears->yaw * pi / 180);
  const float sP = std::sin(ears->pitch * pi / 180), cP = std::cos(ears->pitch * pi / 180);
  const float sR = std::sin(ears->roll * pi / 180), cR = std::cos(ears->roll * pi / 180);
  const float m[3][3] = {{cR * cY - sR * sP * sY, -sR * cP, cR * sY + sR * sP * cY},
                         {sR * cY + cR * sP * sY, cR * cP, sR * sY - cR * sP * cY},
                         {-cP * sY, sP, cP * cY}};
  for (auto& v : ev) {
    const float x = v[0], y = v[1], z = v[2];
    v[0] = x * m[0][0] + y * m[0][1] + z * m[0][2];
    v[1] = x * m[1][0] + y * m[1][1] + z * m[1][2];
    v[2] = x * m[2][0] + y * m[2][1] + z * m[2][2];
  }
  const int nSW = (int)((a.W / 340.0f) * sample_rate), nSH = (int)((a.H / 340.0f) * sample_rate),
            nSL = (int)((a.L / 340.0f) * sample_rate);
  if (nSW <= 0 || nSH <= 0 || nSL <= 0)
    return tanb::rfail(TANB_INVALID_ARG, "room smaller than one sample of sound travel");
  int nW = 1 + length / nSW, nH = 1 + length / nSH, nL = 1 + length / nSL;
  if (flags & TANB_GENROOM_LIMIT_BOUNCES) {
    nW = std::min(nW, max_bounces);
    nH = std::min(nH, max_bounces);
    nL = std::min(nL, max_bounces);
  }
  a.numRefX = 2 * nW;
  a.numRefY = 2 * nH;
  a.numRefZ = 2 * nL;
  // the reference's NDRange: 2n rounded up to the local size 4, ids above 2n return
  auto extent = [](int n2) { return std::min((n2 % 4) ? n2 + 4 - n2 % 4 : n2, n2 + 1); };
  a.cx = extent(a.numRefX);
  a.cy = extent(a.numRefY);
  a.cz = extent(a.numRefZ);
  a.rate = sample_rate;
  a.length = length;
  a.hrtfLength = 2 * (nSW + nSH + nSL);
  a.filterLength = ears->filter_length;
  a.maxGain = 2.0f;
  a.dMin = 2 * es;
  std::memcpy(a.lp, ears->low_pass, sizeof(a.lp));
  std::memcpy(a.hp, ears->high_pass, sizeof(a.hp));
  const long long images = (long long)a.cx * a.cy * a.cz;
  g->images_last = images;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->ctx->device);
  const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((images + 255) / 256, 16LL * sms));
  // calls share the accumulator: each starts after the previous one ended
  e = cudaStreamWaitEvent(st, g->done, 0);
  if (e != cudaSuccess) return tanb::rfail(TANB_FAIL, "%s", cudaGetErrorString(e));
  for (int ch = 0; ch < 2; ++ch) {
    a.hx = ears->head_x + ev[ch][0];
    a.hy = ears->head_y + ev[ch][1];
    a.hz = ears->head_z + ev[ch][2];
    a.evx = ev[2 + ch][0];
    a.evy = ev[2 + ch][1];
    a.evz = ev[2 + ch][2];
    a.earV = std::sqrt(a.evx * a.evx + a.evy * a.evy + a.evz * a.evz);
    unsigned long long* acc = g->acc + (size_t)ch * g->max_length;
    tanb::room_images_kernel<<<blocks, 256, 0, st>>>(a, acc, images);
    tanb::room_fill_kernel<<<(unsigned)std::min(1024, (length + 255) / 256), 256, 0, st>>>(acc, ch ? right : left,
                                                                                         length);
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(g->done, st);
  if (e != cudaSuccess) return tanb::rfail(TANB_FAIL, "room response launch: %s", cudaGetErrorString(e));
  return TANB_OK;
}

int64_t tanb_room_images(tanb_room_generator* g) { return g ? g->images_last : 0; }

int32_t tanb_room_generator_synchronize(tanb_room_generator* g) {
  if (!g) return tanb::rfail(TANB_INVALID_POINTER, "null generator");
  std::lock_guard<std::mutex> lock(g->mu);
  cudaError_t e = cudaSetDevice(g->ctx->device);
  if (e == cudaSuccess) e = cudaEventSynchronize(g->done);
  if (e != cudaSuccess) return tanb::rfail(TANB_FAIL, "%s", cudaGetErrorString(e));
  return TANB_OK;
}

void* tanb_room_generator_stream(tanb_room_generator* g) { return g ? (void*)g->stream : nullptr; }

}  // extern "C"
