// Kernels of the batched engine: every channel of every open session runs in
// one head launch and one persistent tail launch per audio block.
//
//   eng_ir_kernel    one CTA per (IR partition, updated channel): R2C of the
//                    partition, optional FP16/BF16 quantisation with a
//                    power-of-two per-partition scale, stored in the idle slot
//                    (runs on the engine's update stream)
//   eng_head_kernel  one CTA per channel slot: as the single-object head, but
//                    the tail comes from the channel's work-item partial sums
//                    (added in a fixed order) and the delay-line position and
//                    IR slot state live in the device channel table
//   eng_tail_kernel  persistent grid over work items (channel, partition range):
//                    each item streams its partitions of IR spectrum and delay
//                    line once (float4 / uint2 loads) and writes one partial
//                    sum row -- items are of bounded size, so channels with
//                    uneven partition counts balance across the 148 SMs
//
// The per-block sums are the reference's head and tail
// (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:2380-2643);
// the batching across channels with a channel map is the role the reference's
// GPU engine gives processAccum (tan/tanlibrary/src/Graal/GraalConv.cpp:1883-2145).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tanb_engine.h"
#include "tanb_fft.cuh"

namespace tanb {
namespace {

template <int SPEC>
struct SpecT;
template <>
struct SpecT<kSpecFP32> {
  using T = float2;
  static __device__ __forceinline__ float2 get(const void* p, size_t k) { return reinterpret_cast<const float2*>(p)[k]; }
  static __device__ __forceinline__ void put(void* p, size_t k, float2 v) { reinterpret_cast<float2*>(p)[k] = v; }
};
template <>
struct SpecT<kSpecFP16> {
  using T = __half2;
  static __device__ __forceinline__ float2 get(const void* p, size_t k) {
    return __half22float2(reinterpret_cast<const __half2*>(p)[k]);
  }
  static __device__ __forceinline__ void put(void* p, size_t k, float2 v) {
    reinterpret_cast<__half2*>(p)[k] = __float22half2_rn(v);
  }
};
template <>
struct SpecT<kSpecBF16> {
  using T = __nv_bfloat162;
  static __device__ __forceinline__ float2 get(const void* p, size_t k) {
    return __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(p)[k]);
  }
  static __device__ __forceinline__ void put(void* p, size_t k, float2 v) {
    reinterpret_cast<__nv_bfloat162*>(p)[k] = __float22bfloat162_rn(v);
  }
};

__device__ __forceinline__ size_t spec_index(const EngChan& ch, int slot, int part, int B) {
  return ((size_t)slot * ch.P + part) * B;
}

// ---------------------------------------------------------------------------
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_ir_kernel(EngChan* __restrict__ chans, const float* __restrict__ ir, const EngUpd* __restrict__ upd,
                  const float2* __restrict__ tw) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  __shared__ float red[32];
  const int part = blockIdx.x;
  const EngUpd u = upd[blockIdx.y];
  const EngChan ch = chans[u.chan];
  if (part >= ch.P) return;
  const float* h = ir + (size_t)blockIdx.y * u.stride + (size_t)part * M;
  for (int n = threadIdx.x; n < M; n += T)
    sm[n] = (n < M / 2) ? make_float2(h[2 * n], h[2 * n + 1]) : make_float2(0.f, 0.f);
  __syncthreads();
  fft_inplace<LOG2M, false>(sm, tw);
  // split step in place: thread owning pair (k, M-k) writes both
  for (int k = threadIdx.x; k <= M / 2; k += T) {
    if (k == 0) {
      sm[0] = rfft_post_dc(sm[0]);
    } else {
      const int km = M - k;
      const float2 a = sm[k], b = sm[km];
      const float2 Xk = rfft_post(a, b, __ldg(tw + k));
      const float2 Xm = rfft_post(b, a, __ldg(tw + km));
      sm[k] = Xk;
      if (km != k) sm[km] = Xm;
    }
  }
  __syncthreads();
  float scale = 1.0f;
  if constexpr (SPEC != kSpecFP32) {
    float mx = 0.f;
    for (int k = threadIdx.x; k < M; k += T) mx = fmaxf(mx, fmaxf(fabsf(sm[k].x), fabsf(sm[k].y)));
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
      mx = (threadIdx.x < (T + 31) / 32) ? red[threadIdx.x] : 0.f;
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (threadIdx.x == 0) red[0] = mx;
    }
    __syncthreads();
    mx = red[0];
    // power of two with the largest magnitude mapped to [2^14, 2^15)
    int e = 0;
    if (mx > 0.f) {
      frexpf(mx, &e);  // mx = f * 2^e, f in [0.5, 1)
      e -= 15;
    }
    scale = ldexpf(1.0f, e);
    if (threadIdx.x == 0) ch.scale[(size_t)u.slot * ch.P + part] = scale;
  }
  const float inv = 1.0f / scale;  // exact: power of two
  for (int k = threadIdx.x; k < M; k += T)
    SpecT<SPEC>::put(ch.H, spec_index(ch, u.slot, part, M) + k, make_float2(sm[k].x * inv, sm[k].y * inv));
}

// ---------------------------------------------------------------------------
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_head_kernel(EngChan* __restrict__ chans, const float* __restrict__ in_base, float* __restrict__ out_base,
                    int ld, const float2* __restrict__ tw) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  float2* z = sm;
  float2* z2 = sm + M;
  const int c = blockIdx.x;
  const EngChan ch = chans[c];
  if (!ch.run) return;
  const bool swap = ch.pending != 0;
  const int P = ch.P;
  const int cur = (ch.cur - 1 + P) % P;
  const int slot_old = ch.active, slot_new = 1 - ch.active;
  const float* x = in_base ? in_base + (size_t)c * ld : nullptr;
  float* y = out_base + (size_t)c * ld;

  for (int n = threadIdx.x; n < M; n += T) {
    const float* src = (n < M / 2) ? ch.prev + 2 * n : (x ? x + 2 * (n - M / 2) : nullptr);
    z[n] = src ? make_float2(src[0], src[1]) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (int n = threadIdx.x; n < M / 2; n += T) reinterpret_cast<float2*>(ch.prev)[n] = z[n + M / 2];
  fft_inplace<LOG2M, false>(z, tw);

  float2* F = ch.fdl + (size_t)cur * M;
  const size_t h0 = spec_index(ch, slot_old, 0, M);
  const size_t h1 = spec_index(ch, slot_new, 0, M);
  float s0 = 1.f, s1 = 1.f;
  if constexpr (SPEC != kSpecFP32) {
    s0 = ch.scale[(size_t)slot_old * P];
    s1 = ch.scale[(size_t)slot_new * P];
  }
  const float inv_n = 1.0f / (float)(2 * M);
  const float2* part0 = ch.part;
  const float2* part1 = ch.part + (size_t)ch.nitem * M;
  for (int k = threadIdx.x; k <= M / 2; k += T) {
    const int km = (k == 0) ? 0 : M - k;
    // tails: partial sums of the work items, in item order
    float2 tk = make_float2(0.f, 0.f), tm = tk, uk = tk, um = tk;
    for (int r = 0; r < ch.nitem; ++r) {
      const float2 a = part0[(size_t)r * M + k], b = part0[(size_t)r * M + km];
      tk.x += a.x; tk.y += a.y;
      tm.x += b.x; tm.y += b.y;
      if (swap) {
        const float2 a1 = part1[(size_t)r * M + k], b1 = part1[(size_t)r * M + km];
        uk.x += a1.x; uk.y += a1.y;
        um.x += b1.x; um.y += b1.y;
      }
    }
    if (k == 0) {
      const float2 X = rfft_post_dc(z[0]);
      F[0] = X;
      float2 hh = SpecT<SPEC>::get(ch.H, h0);
      hh.x *= s0; hh.y *= s0;
      z[0] = irfft_pre_dc(c_mac_dc(tk, X, hh), inv_n);
      if (swap) {
        float2 hn = SpecT<SPEC>::get(ch.H, h1);
        hn.x *= s1; hn.y *= s1;
        z2[0] = irfft_pre_dc(c_mac_dc(uk, X, hn), inv_n);
      }
    } else {
      const float2 wk = __ldg(tw + k), wm = __ldg(tw + km);
      const float2 a = z[k], b = z[km];
      const float2 Xk = rfft_post(a, b, wk);
      const float2 Xm = rfft_post(b, a, wm);
      F[k] = Xk;
      if (km != k) F[km] = Xm;
      float2 hk = SpecT<SPEC>::get(ch.H, h0 + k), hm = SpecT<SPEC>::get(ch.H, h0 + km);
      hk.x *= s0; hk.y *= s0; hm.x *= s0; hm.y *= s0;
      const float2 Ak = c_mac(tk, Xk, hk);
      const float2 Am = c_mac(tm, Xm, hm);
      z[k] = irfft_pre(Ak, Am, wk, inv_n);
      if (km != k) z[km] = irfft_pre(Am, Ak, wm, inv_n);
      if (swap) {
        float2 gk = SpecT<SPEC>::get(ch.H, h1 + k), gm = SpecT<SPEC>::get(ch.H, h1 + km);
        gk.x *= s1; gk.y *= s1; gm.x *= s1; gm.y *= s1;
        const float2 Bk = c_mac(uk, Xk, gk);
        const float2 Bm = c_mac(um, Xm, gm);
        z2[k] = irfft_pre(Bk, Bm, wk, inv_n);
        if (km != k) z2[km] = irfft_pre(Bm, Bk, wm, inv_n);
      }
    }
  }
  __syncthreads();
  fft_inplace<LOG2M, true>(z, tw);
  if (swap) fft_inplace<LOG2M, true>(z2, tw);
  const float step = 1.0f / (float)M;
  for (int m = M / 2 + threadIdx.x; m < M; m += T) {
    const int i = 2 * (m - M / 2);
    const float2 yo = z[m];
    if (!swap) {
      y[i] = yo.x;
      y[i + 1] = yo.y;
    } else {
      const float2 yn = z2[m];
      y[i] = yn.x * (step * (float)i) + yo.x * (step * (float)(M - i));
      y[i + 1] = yn.y * (step * (float)(i + 1)) + yo.y * (step * (float)(M - i - 1));
    }
  }
  if (threadIdx.x == 0) {
    chans[c].cur = cur;
    if (swap) {
      chans[c].active = slot_new;
      chans[c].pending = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Two packed bins per thread. FDL rows are float4 pairs; spectra are float4
// (FP32) or uint2 (two half2 / bfloat162) pairs.
template <int SPEC>
__device__ __forceinline__ void load_h2(const void* H, size_t idx2, float2& a, float2& b) {
  if constexpr (SPEC == kSpecFP32) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(H) + idx2);
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
  } else {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(H) + idx2);
    if constexpr (SPEC == kSpecFP16) {
      a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
      b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    } else {
      a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
      b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
    }
  }
}

template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(1 << (LOG2M - 1))
    eng_tail_kernel(const EngChan* __restrict__ chans, const EngItem* __restrict__ items, int item0, int nitems,
                    int mode) {
  constexpr int M = 1 << LOG2M;
  constexpr int U = M / 2;  // threads = pairs of bins
  const int u = threadIdx.x;
  for (int it = item0 + blockIdx.x; it < item0 + nitems; it += gridDim.x) {
    const EngItem w = items[it];
    if (w.chan < 0) continue;
    const EngChan ch = chans[w.chan];
    if (mode == 0 ? !ch.run : !ch.pending) continue;
    const int P = ch.P;
    const int slot = (mode == 0) ? ch.active : 1 - ch.active;
    // delay-line slot of partition i for the next block: (cur + i - 1) mod P
    int fs = (ch.cur + w.i0 - 1) % P;
    const float4* Fc = reinterpret_cast<const float4*>(ch.fdl) + u;
    const size_t hbase2 = (((size_t)slot * P) * M) / 2 + u;  // in bin pairs
    const float* sc = (SPEC != kSpecFP32) ? ch.scale + (size_t)slot * P : nullptr;
    const bool dc = (u == 0);
    float2 acc0 = make_float2(0.f, 0.f), acc1 = acc0;
    int i = w.i0;
    for (; i + 4 <= w.i1; i += 4) {
      float4 f[4];
      float2 ha[4], hb[4];
      float s[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        f[q] = __ldg(Fc + (size_t)fs * U);
        load_h2<SPEC>(ch.H, hbase2 + (size_t)(i + q) * U, ha[q], hb[q]);
        s[q] = (SPEC != kSpecFP32) ? __ldg(sc + i + q) : 1.f;
        fs = (fs + 1 == P) ? 0 : fs + 1;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (SPEC != kSpecFP32) {
          ha[q].x *= s[q]; ha[q].y *= s[q]; hb[q].x *= s[q]; hb[q].y *= s[q];
        }
        const float2 fa = make_float2(f[q].x, f[q].y), fb = make_float2(f[q].z, f[q].w);
        acc0 = dc ? c_mac_dc(acc0, fa, ha[q]) : c_mac(acc0, fa, ha[q]);
        acc1 = c_mac(acc1, fb, hb[q]);
      }
    }
    for (; i < w.i1; ++i) {
      const float4 f = __ldg(Fc + (size_t)fs * U);
      float2 ha, hb;
      load_h2<SPEC>(ch.H, hbase2 + (size_t)i * U, ha, hb);
      if (SPEC != kSpecFP32) {
        const float s = __ldg(sc + i);
        ha.x *= s; ha.y *= s; hb.x *= s; hb.y *= s;
      }
      fs = (fs + 1 == P) ? 0 : fs + 1;
      const float2 fa = make_float2(f.x, f.y), fb = make_float2(f.z, f.w);
      acc0 = dc ? c_mac_dc(acc0, fa, ha) : c_mac(acc0, fa, ha);
      acc1 = c_mac(acc1, fb, hb);
    }
    float4* dst = reinterpret_cast<float4*>(ch.part + ((size_t)mode * ch.nitem + w.row) * M);
    dst[u] = make_float4(acc0.x, acc0.y, acc1.x, acc1.y);
  }
}

template <int LOG2M, int SPEC>
cudaError_t attrs_t() {
  const int smem = 2 * (1 << LOG2M) * (int)sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(eng_head_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(eng_ir_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem / 2);
}

template <int LOG2M>
cudaError_t attrs_all() {
  cudaError_t e;
  if ((e = attrs_t<LOG2M, kSpecFP32>()) != cudaSuccess) return e;
  if ((e = attrs_t<LOG2M, kSpecFP16>()) != cudaSuccess) return e;
  return attrs_t<LOG2M, kSpecBF16>();
}

template <int LOG2M, int SPEC>
cudaError_t ir_t(EngChan* chans, const float* ir, const EngUpd* upd, int nupd, int maxP, const float2* tw,
                 cudaStream_t st) {
  using S = FftShape<LOG2M>;
  dim3 grid(maxP, nupd);
  eng_ir_kernel<LOG2M, SPEC><<<grid, S::T, S::M * sizeof(float2), st>>>(chans, ir, upd, tw);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t head_t(EngChan* chans, int nslots, const float* in, float* out, int ld, const float2* tw,
                   cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_head_kernel<LOG2M, SPEC><<<nslots, S::T, 2 * S::M * sizeof(float2), st>>>(chans, in, out, ld, tw);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t tail_t(const EngChan* chans, const EngItem* items, int item0, int nitems, int mode, int grid,
                   cudaStream_t st) {
  eng_tail_kernel<LOG2M, SPEC><<<grid, 1 << (LOG2M - 1), 0, st>>>(chans, items, item0, nitems, mode);
  return cudaGetLastError();
}

#define ENG_DISPATCH(L2, SP, FN, ...)                                     \
  switch ((L2) * 4 + (SP)) {                                              \
    case 7 * 4 + 0: return FN<7, 0>(__VA_ARGS__);                         \
    case 7 * 4 + 1: return FN<7, 1>(__VA_ARGS__);                         \
    case 7 * 4 + 2: return FN<7, 2>(__VA_ARGS__);                         \
    case 8 * 4 + 0: return FN<8, 0>(__VA_ARGS__);                         \
    case 8 * 4 + 1: return FN<8, 1>(__VA_ARGS__);                         \
    case 8 * 4 + 2: return FN<8, 2>(__VA_ARGS__);                         \
    case 9 * 4 + 0: return FN<9, 0>(__VA_ARGS__);                         \
    case 9 * 4 + 1: return FN<9, 1>(__VA_ARGS__);                         \
    case 9 * 4 + 2: return FN<9, 2>(__VA_ARGS__);                         \
    case 10 * 4 + 0: return FN<10, 0>(__VA_ARGS__);                       \
    case 10 * 4 + 1: return FN<10, 1>(__VA_ARGS__);                       \
    case 10 * 4 + 2: return FN<10, 2>(__VA_ARGS__);                       \
    case 11 * 4 + 0: return FN<11, 0>(__VA_ARGS__);                       \
    case 11 * 4 + 1: return FN<11, 1>(__VA_ARGS__);                       \
    case 11 * 4 + 2: return FN<11, 2>(__VA_ARGS__);                       \
    default: return cudaErrorInvalidValue;                                \
  }

}  // namespace

cudaError_t eng_prepare() {
  static cudaError_t r = [] {
    cudaError_t e;
    if ((e = attrs_all<7>()) != cudaSuccess) return e;
    if ((e = attrs_all<8>()) != cudaSuccess) return e;
    if ((e = attrs_all<9>()) != cudaSuccess) return e;
    if ((e = attrs_all<10>()) != cudaSuccess) return e;
    return attrs_all<11>();
  }();
  return r;
}

cudaError_t eng_launch_ir(int log2B, int spec, EngChan* chans, const float* ir, const EngUpd* upd, int nupd,
                          int maxP, const float2* tw, cudaStream_t st) {
  if (nupd <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, ir_t, chans, ir, upd, nupd, maxP, tw, st);
}

cudaError_t eng_launch_head(int log2B, int spec, EngChan* chans, int nslots, const float* in, float* out, int ld,
                            const float2* tw, cudaStream_t st) {
  if (nslots <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, head_t, chans, nslots, in, out, ld, tw, st);
}

cudaError_t eng_launch_tail(int log2B, int spec, const EngChan* chans, const EngItem* items, int item0,
                            int nitems, int mode, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, tail_t, chans, items, item0, nitems, mode, grid, st);
}

}  // namespace tanb
