// TIME_DOMAIN method: direct FIR over a per-channel circular history, the GPU
// form of ProcessDirect / ovlTimeDomainCPU
// (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:721-762,
// 2757-2782; the reference's OpenCL kernel is TimeDomainConvolution.cl:234-273,
// launched with one work-item per work-group).
//
//   td_insert_kernel  hist[c][(pos + i) mod len] = in[c][i], i < n
//   td_fir_kernel     out[c][j] = sum_{k=first}^{last-1} hist[c][(pos + j - k) mod len] * ir[c][k]
//
// The FIR kernel tiles 1024 outputs x 512 taps per step in shared memory: the
// IR chunk and the history window (1024 + 512 - 1 samples, gathered with the
// circular wrap) are staged once, then each thread slides a 4-sample register
// window down the history, one shared load and four FMAs per tap. Taps are
// accumulated in increasing k with fused multiply-adds, the order of the
// reference's loop. On a crossfade block a second IR is convolved and the two
// outputs blended with the reference's weights (ConvolutionImpl.cpp:1392-1408).
#include "tanb_internal.h"

namespace tanb {
namespace {

constexpr int kTJ = 1024;    // outputs per CTA
constexpr int kTK = 512;     // taps per shared-memory chunk
constexpr int kThreads = 256;
constexpr int kPerThread = kTJ / kThreads;  // 4

__global__ void td_insert_kernel(float* hist, int len, const TdChan* __restrict__ ch, int n) {
  const int c = blockIdx.y;
  const TdChan t = ch[c];
  if (!t.run || !t.in) return;
  float* h = hist + (size_t)c * len;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    h[(int)(((long long)t.pos + i) % len)] = t.in[i];
}

__device__ __forceinline__ void fir_tile(const float* __restrict__ h, int len, int pos, const float* __restrict__ ir,
                                         int first, int last, int j0, float* xs, float* ws, float acc[kPerThread]) {
  const int tid = threadIdx.x;
  const int jt = j0 + tid * kPerThread;  // first output of this thread
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) acc[q] = 0.f;
  for (int k0 = first; k0 < last; k0 += kTK) {
    const int kn = min(kTK, last - k0);
    __syncthreads();
    for (int k = tid; k < kTK; k += kThreads) ws[k] = (k < kn) ? ir[k0 + k] : 0.f;
    // window covers history offsets (j0 - k0 - kTK + 1) .. (j0 + kTJ - 1 - k0)
    const int base = j0 - k0 - kTK + 1;
    for (int i = tid; i < kTJ + kTK - 1; i += kThreads) {
      long long a = (long long)pos + base + i;
      a %= len;
      if (a < 0) a += len;
      xs[i] = h[a];
    }
    __syncthreads();
    // output jt+q, tap k0+k reads window index (jt + q - j0) - k + kTK - 1
    const int w0 = (jt - j0) + kTK - 1;
    float win[kPerThread];
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) win[q] = xs[w0 + q];
    for (int k = 0; k < kn; ++k) {
      const float w = ws[k];
#pragma unroll
      for (int q = 0; q < kPerThread; ++q) acc[q] = __fmaf_rn(win[q], w, acc[q]);
#pragma unroll
      for (int q = kPerThread - 1; q > 0; --q) win[q] = win[q - 1];
      if (k + 1 < kn) win[0] = xs[w0 - k - 1];
    }
  }
}

__global__ void __launch_bounds__(kThreads) td_fir_kernel(const float* hist, int len, const TdChan* __restrict__ ch,
                                                        int n, int fade_len) {
  __shared__ float xs[kTJ + kTK];
  __shared__ float ws[kTK];
  const int c = blockIdx.y;
  const TdChan t = ch[c];
  if (!t.run) return;
  const int j0 = blockIdx.x * kTJ;
  const float* h = hist + (size_t)c * len;
  float a[kPerThread];
  fir_tile(h, len, t.pos, t.ir, t.first, t.last, j0, xs, ws, a);
  float b[kPerThread];
  if (t.swap) fir_tile(h, len, t.pos, t.ir_new, t.first, t.last, j0, xs, ws, b);
  if (!t.out) return;
  const float step = 1.0f / (float)fade_len;
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int j = j0 + threadIdx.x * kPerThread + q;
    if (j >= n) continue;
    if (!t.swap || t.fade0 + j >= fade_len) {
      t.out[j] = t.swap ? b[q] : a[q];
    } else {
      const float w1 = step * (float)(t.fade0 + j), w2 = step * (float)(fade_len - t.fade0 - j);
      t.out[j] = b[q] * w1 + a[q] * w2;
    }
  }
}

}  // namespace

cudaError_t launch_td(float* hist, int len, const TdChan* ch, int C, int n, int fade_len, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  dim3 gi((n + 255) / 256, C);
  td_insert_kernel<<<gi, 256, 0, st>>>(hist, len, ch, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 gf((n + kTJ - 1) / kTJ, C);
  td_fir_kernel<<<gf, kThreads, 0, st>>>(hist, len, ch, n, fade_len);
  return cudaGetLastError();
}

}  // namespace tanb
