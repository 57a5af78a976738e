// sm_100a kernels of the uniformly-partitioned overlap-save convolution.
//
//   ir_spectrum_kernel  one CTA per (IR partition, channel): R2C of [h_i, 0^B]
//   head_kernel         one CTA per channel: R2C of [x_{k-1}, x_k] into the
//                       delay line, MAC with partition 0, add the precomputed
//                       tail, C2R, output the upper B samples (crossfading old
//                       and new IR on a swap block)
//   tail_kernel         streaming MAC over partitions 1..P-1 for the next block
//                       (the HBM-bound kernel): float4 loads of the IR spectrum
//                       and the delay line, partitions split across warps and
//                       reduced in shared memory in a fixed order
//
// The reference computes the same sums on the CPU with an overlap-add form
// (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:2380-2643);
// overlap-save needs no overlap buffer and gives the exact new-IR output on a
// swap block from the same delay line.
#include <cmath>

#include "tanb_fft.cuh"
#include "tanb_internal.h"

namespace tanb {
namespace {


template <int LOG2M>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    ir_spectrum_kernel(DevState s, const float* __restrict__ ir, const int* __restrict__ chans,
                       const ChanCtl* __restrict__ ctl) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  const int part = blockIdx.x;
  const int row = blockIdx.y;
  const int c = chans[row];
  const int slot = ctl[c].slot_new;
  const float* h = ir + (size_t)row * s.P * M + (size_t)part * M;
  for (int n = threadIdx.x; n < M; n += T)
    sm[n] = (n < M / 2) ? make_float2(h[2 * n], h[2 * n + 1]) : make_float2(0.f, 0.f);
  __syncthreads();
  fft_inplace<LOG2M, false>(sm, s.tw);
  float2* H = s.H + h_index(s, c, slot, part);
  for (int k = threadIdx.x; k <= M / 2; k += T) {
    if (k == 0) {
      H[0] = rfft_post_dc(sm[0]);
    } else {
      const int km = M - k;
      const float2 a = sm[k], b = sm[km];
      H[k] = rfft_post(a, b, __ldg(s.tw + k));
      if (km != k) H[km] = rfft_post(b, a, __ldg(s.tw + km));
    }
  }
}

template <int LOG2M>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    head_kernel(DevState s, const ChanCtl* __restrict__ ctl, const float* const* __restrict__ inp,
                float* const* __restrict__ outp, int cur) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  float2* z = sm;       // old / only IR
  float2* z2 = sm + M;  // new IR on a swap block
  const int c = blockIdx.x;
  const ChanCtl cc = ctl[c];
  if (!cc.run) return;
  const bool swap = cc.swap != 0;
  const float* x = inp[c];
  float* y = outp[c];
  float* prev = s.prev + (size_t)c * M;

  // frame [x_{k-1}, x_k] packed as complex pairs
  for (int n = threadIdx.x; n < M; n += T) {
    const float* src = (n < M / 2) ? prev + 2 * n : (x ? x + 2 * (n - M / 2) : nullptr);
    z[n] = src ? make_float2(src[0], src[1]) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (int n = threadIdx.x; n < M / 2; n += T) reinterpret_cast<float2*>(prev)[n] = z[n + M / 2];

  fft_inplace<LOG2M, false>(z, s.tw);

  float2* F = s.fdl + ((size_t)c * s.P + cur) * M;
  const float2* h0 = s.H + h_index(s, c, cc.slot_cur, 0);
  const float2* h1 = s.H + h_index(s, c, cc.slot_new, 0);
  const float2* t0 = s.tail + (size_t)c * 2 * M;
  const float2* t1 = t0 + M;
  const float inv_n = 1.0f / (float)(2 * M);
  for (int k = threadIdx.x; k <= M / 2; k += T) {
    if (k == 0) {
      const float2 X = rfft_post_dc(z[0]);
      F[0] = X;
      z[0] = irfft_pre_dc(c_mac_dc(t0[0], X, h0[0]), inv_n);
      if (swap) z2[0] = irfft_pre_dc(c_mac_dc(t1[0], X, h1[0]), inv_n);
    } else {
      const int km = M - k;
      const float2 wk = __ldg(s.tw + k), wm = __ldg(s.tw + km);
      const float2 a = z[k], b = z[km];
      const float2 Xk = rfft_post(a, b, wk);
      const float2 Xm = rfft_post(b, a, wm);
      F[k] = Xk;
      if (km != k) F[km] = Xm;
      const float2 Ak = c_mac(t0[k], Xk, h0[k]);
      const float2 Am = c_mac(t0[km], Xm, h0[km]);
      z[k] = irfft_pre(Ak, Am, wk, inv_n);
      if (km != k) z[km] = irfft_pre(Am, Ak, wm, inv_n);
      if (swap) {
        const float2 Bk = c_mac(t1[k], Xk, h1[k]);
        const float2 Bm = c_mac(t1[km], Xm, h1[km]);
        z2[k] = irfft_pre(Bk, Bm, wk, inv_n);
        if (km != k) z2[km] = irfft_pre(Bm, Bk, wm, inv_n);
      }
    }
  }
  __syncthreads();
  fft_inplace<LOG2M, true>(z, s.tw);
  if (swap) fft_inplace<LOG2M, true>(z2, s.tw);

  // overlap-save: samples [B, 2B) of the circular result are the output
  if (!y) return;
  const float step = 1.0f / (float)M;
  for (int m = M / 2 + threadIdx.x; m < M; m += T) {
    const int i = 2 * (m - M / 2);
    const float2 yo = z[m];
    if (!swap) {
      y[i] = yo.x;
      y[i + 1] = yo.y;
    } else {
      const float2 yn = z2[m];
      const float a0 = step * (float)i, b0 = step * (float)(M - i);
      const float a1 = step * (float)(i + 1), b1 = step * (float)(M - i - 1);
      y[i] = yn.x * a0 + yo.x * b0;
      y[i + 1] = yn.y * a1 + yo.y * b1;
    }
  }
}

// One float4 = two packed bins. u == 0 holds the packed (DC, Nyquist) pair.
__device__ __forceinline__ float4 mac4(float4 acc, float4 f, float4 h, bool dc) {
  float2 lo = dc ? c_mac_dc(make_float2(acc.x, acc.y), make_float2(f.x, f.y), make_float2(h.x, h.y))
                 : c_mac(make_float2(acc.x, acc.y), make_float2(f.x, f.y), make_float2(h.x, h.y));
  float2 hi = c_mac(make_float2(acc.z, acc.w), make_float2(f.z, f.w), make_float2(h.z, h.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

template <int UX, int SY>
__global__ void __launch_bounds__(UX* SY)
    tail_kernel(DevState s, const ChanCtl* __restrict__ ctl, int which, int cur) {
  const int c = blockIdx.y;
  const ChanCtl cc = ctl[c];
  if (which == 0 ? !cc.run : !cc.swap) return;
  const int slot = (which == 0) ? (cc.swap ? cc.slot_new : cc.slot_cur) : cc.slot_new;
  const int U = s.B >> 1;  // float4 units per partition
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int u = blockIdx.x * UX + tx;
  const int P = s.P;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (u < U && P > 1) {
    const float4* Hc = reinterpret_cast<const float4*>(s.H + h_index(s, c, slot, 0)) + u;
    const float4* Fc = reinterpret_cast<const float4*>(s.fdl + (size_t)c * P * s.B) + u;
    const int nparts = P - 1;
    const int chunk = (nparts + SY - 1) / SY;
    const int i0 = 1 + ty * chunk;
    const int i1 = min(P, i0 + chunk);
    int fs = (cur + i0 - 1) % P;
    const bool dc = (u == 0);
    int i = i0;
    for (; i + 4 <= i1; i += 4) {
      float4 h[4], f[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        h[q] = __ldg(Hc + (size_t)(i + q) * U);
        f[q] = __ldg(Fc + (size_t)fs * U);
        fs = (fs + 1 == P) ? 0 : fs + 1;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) acc = mac4(acc, f[q], h[q], dc);
    }
    for (; i < i1; ++i) {
      const float4 h = __ldg(Hc + (size_t)i * U);
      const float4 f = __ldg(Fc + (size_t)fs * U);
      fs = (fs + 1 == P) ? 0 : fs + 1;
      acc = mac4(acc, f, h, dc);
    }
  }
  if constexpr (SY > 1) {
    __shared__ float4 red[SY][UX];
    red[ty][tx] = acc;
    __syncthreads();
    if (ty != 0) return;
#pragma unroll
    for (int q = 1; q < SY; ++q) {
      const float4 r = red[q][tx];
      acc.x += r.x;
      acc.y += r.y;
      acc.z += r.z;
      acc.w += r.w;
    }
  }
  if (u < U) reinterpret_cast<float4*>(s.tail + ((size_t)c * 2 + which) * s.B)[u] = acc;
}

template <int LOG2M>
cudaError_t set_attrs() {
  const int smem = 2 * (1 << LOG2M) * (int)sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(head_kernel<LOG2M>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(ir_spectrum_kernel<LOG2M>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem / 2);
}

template <int LOG2M>
cudaError_t launch_ir_t(const DevState& s, const float* ir, const int* chans, int nch, const ChanCtl* ctl,
                        cudaStream_t st) {
  using S = FftShape<LOG2M>;
  dim3 grid(s.P, nch);
  ir_spectrum_kernel<LOG2M><<<grid, S::T, S::M * sizeof(float2), st>>>(s, ir, chans, ctl);
  return cudaGetLastError();
}

template <int LOG2M>
cudaError_t launch_head_t(const DevState& s, const ChanCtl* ctl, const float* const* in, float* const* out,
                          int cur, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  head_kernel<LOG2M><<<s.C, S::T, 2 * S::M * sizeof(float2), st>>>(s, ctl, in, out, cur);
  return cudaGetLastError();
}

#define TANB_DISPATCH_LOG2(L2, FN, ...)                          \
  switch (L2) {                                                  \
    case 5: return FN<5>(__VA_ARGS__);                           \
    case 6: return FN<6>(__VA_ARGS__);                           \
    case 7: return FN<7>(__VA_ARGS__);                           \
    case 8: return FN<8>(__VA_ARGS__);                           \
    case 9: return FN<9>(__VA_ARGS__);                           \
    case 10: return FN<10>(__VA_ARGS__);                         \
    case 11: return FN<11>(__VA_ARGS__);                         \
    case 12: return FN<12>(__VA_ARGS__);                         \
    case 13: return FN<13>(__VA_ARGS__);                         \
    default: return cudaErrorInvalidValue;                       \
  }

template <int UX, int SY>
cudaError_t launch_tail_t(const DevState& s, const ChanCtl* ctl, int which, int cur, cudaStream_t st) {
  const int U = s.B >> 1;
  dim3 grid((U + UX - 1) / UX, s.C);
  dim3 block(UX, SY);
  tail_kernel<UX, SY><<<grid, block, 0, st>>>(s, ctl, which, cur);
  return cudaGetLastError();
}

}  // namespace

cudaError_t prepare_kernels() {
  static cudaError_t result = [] {
    cudaError_t e;
    if ((e = set_attrs<5>()) != cudaSuccess) return e;
    if ((e = set_attrs<6>()) != cudaSuccess) return e;
    if ((e = set_attrs<7>()) != cudaSuccess) return e;
    if ((e = set_attrs<8>()) != cudaSuccess) return e;
    if ((e = set_attrs<9>()) != cudaSuccess) return e;
    if ((e = set_attrs<10>()) != cudaSuccess) return e;
    if ((e = set_attrs<11>()) != cudaSuccess) return e;
    if ((e = set_attrs<12>()) != cudaSuccess) return e;
    return set_attrs<13>();
  }();
  return result;
}

cudaError_t launch_ir_spectrum(const DevState& s, const float* ir, const int* chans, int nch,
                               const ChanCtl* ctl, cudaStream_t st) {
  if (nch <= 0) return cudaSuccess;
  TANB_DISPATCH_LOG2(s.log2B, launch_ir_t, s, ir, chans, nch, ctl, st);
}

cudaError_t launch_head_ptrs(const DevState& s, const ChanCtl* ctl, const float* const* in,
                             float* const* out, int cur, cudaStream_t st) {
  TANB_DISPATCH_LOG2(s.log2B, launch_head_t, s, ctl, in, out, cur, st);
}

cudaError_t launch_tail(const DevState& s, const ChanCtl* ctl, int which, int cur, MacTiling t,
                        cudaStream_t st) {
  if (s.P <= 1) return cudaSuccess;
  if (t.ux == 16 && t.sy == 16) return launch_tail_t<16, 16>(s, ctl, which, cur, st);
  if (t.ux == 32 && t.sy == 8) return launch_tail_t<32, 8>(s, ctl, which, cur, st);
  if (t.ux == 64 && t.sy == 4) return launch_tail_t<64, 4>(s, ctl, which, cur, st);
  if (t.ux == 128 && t.sy == 2) return launch_tail_t<128, 2>(s, ctl, which, cur, st);
  if (t.ux == 32 && t.sy == 16) return launch_tail_t<32, 16>(s, ctl, which, cur, st);
  if (t.ux == 64 && t.sy == 8) return launch_tail_t<64, 8>(s, ctl, which, cur, st);
  return cudaErrorInvalidValue;
}

void make_twiddles(int N, float2* out) {
  const int q4 = N / 4;
  for (int j = 0; j < N; ++j) {
    const int q = j / q4, r = j % q4;
    const double th = 2.0 * M_PI * (double)r / (double)N;
    const double c = std::cos(th), sn = std::sin(th);
    double cc, ss;  // cos and sin of 2 pi j / N
    switch (q) {
      case 0: cc = c; ss = sn; break;
      case 1: cc = -sn; ss = c; break;
      case 2: cc = -c; ss = -sn; break;
      default: cc = sn; ss = -c; break;
    }
    out[j] = make_float2((float)cc, (float)(-ss));
  }
}

}  // namespace tanb
