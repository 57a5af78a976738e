// Kernels of the batched engine: every channel of every open session runs in
// ONE launch per audio block.
//
//   eng_ir_kernel      one CTA per (IR partition, updated channel): R2C of the
//                      partition, optional FP16/BF16 quantisation with a
//                      power-of-two per-partition scale, stored in the idle slot
//                      (runs on the engine's update stream)
//   eng_block_kernel   per block: the first CTAs are a persistent grid over
//                      work items (channel, partition range within [2, P))
//                      writing the partial sums of the NEXT block; the last
//                      nslots CTAs are the heads of the channel slots (as the
//                      single-object head, with the tail from the channel's
//                      partial-sum rows plus the partition-1 product computed
//                      here), dispatched into the slots the items leave. Items
//                      read only delay-line slots X_{k-1} and older, which no
//                      head writes, and write the other parity's rows, which no
//                      head reads, so heads and tail items run side by side in
//                      one grid with no dependency between them. Channel state
//                      (delay-line position, IR slots) is read by every CTA as
//                      it was at launch; the last CTA to finish advances it.
//   eng_commit_kernel  partial sums of a newly committed IR for the coming block
//                      (before that block's launch), from the current delay line
//
// The per-block sums are the reference's head and tail
// (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:2380-2643);
// the batching across channels with a channel map is the role the reference's
// GPU engine gives processAccum (tan/tanlibrary/src/Graal/GraalConv.cpp:1883-2145).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "tanb_engine.h"
#include "tanb_fft.cuh"
#include "tanb_internal.h"

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

// FP16 / BF16 spectra carry a power-of-two scale per partition.
template <int SPEC>
constexpr bool kScaled = SPEC == kSpecFP16 || SPEC == kSpecBF16;

// 24-bit storage (kSpecFP24): an FP32 value with its mantissa rounded to
// nearest even at 15 bits (sign, 8-bit exponent, 15-bit fraction). A row of M
// packed bins is a plane of M uint32 (the upper 16 bits of re and im) followed
// by a plane of M uint16 (the next 8 bits of re and im): 6 M bytes, aligned
// 8- and 4-byte loads for two bins. Used for IR spectra and delay-line rows.
__device__ __forceinline__ unsigned f24_encode(float f) {
  const unsigned u = __float_as_uint(f);
  return (u + 0x7Fu + ((u >> 8) & 1u)) >> 8;
}
__device__ __forceinline__ float f24_decode(unsigned hi16, unsigned lo8) {
  return __uint_as_float((hi16 << 16) | (lo8 << 8));
}
template <int M>
__device__ __forceinline__ float2 f24_bin(const void* row, int k) {
  const unsigned hi = reinterpret_cast<const unsigned*>(row)[k];
  const unsigned lo = reinterpret_cast<const unsigned short*>(static_cast<const char*>(row) + 4 * M)[k];
  return make_float2(f24_decode(hi & 0xFFFFu, lo & 0xFFu), f24_decode(hi >> 16, lo >> 8));
}
template <int M>
__device__ __forceinline__ void f24_put(void* row, int k, float2 v) {
  const unsigned re = f24_encode(v.x), im = f24_encode(v.y);
  reinterpret_cast<unsigned*>(row)[k] = (re >> 8) | ((im >> 8) << 16);
  reinterpret_cast<unsigned short*>(static_cast<char*>(row) + 4 * M)[k] =
      (unsigned short)((re & 0xFFu) | ((im & 0xFFu) << 8));
}
// bins 2u and 2u + 1
template <int M>
__device__ __forceinline__ void f24_unit(const void* row, int u, float2& a, float2& b) {
  const uint2 hi = __ldg(reinterpret_cast<const uint2*>(row) + u);
  const unsigned lo = __ldg(reinterpret_cast<const unsigned*>(static_cast<const char*>(row) + 4 * M) + u);
  a = make_float2(f24_decode(hi.x & 0xFFFFu, lo & 0xFFu), f24_decode(hi.x >> 16, (lo >> 8) & 0xFFu));
  b = make_float2(f24_decode(hi.y & 0xFFFFu, (lo >> 16) & 0xFFu), f24_decode(hi.y >> 16, lo >> 24));
}
template <int M>
__device__ __forceinline__ const void* f24_row(const void* base, size_t row) {
  return static_cast<const char*>(base) + row * (size_t)(6 * M);
}
template <int M>
__device__ __forceinline__ void* f24_row(void* base, size_t row) {
  return static_cast<char*>(base) + row * (size_t)(6 * M);
}

// Delay-line slot rows: FP32 float2[M], or 24-bit rows with kSpecFP24.
template <int SPEC, int M>
__device__ __forceinline__ float2 x_bin(const float2* fdl, int slot, int k) {
  if constexpr (SPEC == kSpecFP24) return f24_bin<M>(f24_row<M>(fdl, slot), k);
  else return fdl[(size_t)slot * M + k];
}
template <int SPEC, int M>
__device__ __forceinline__ void x_put(float2* fdl, int slot, int k, float2 v) {
  if constexpr (SPEC == kSpecFP24) f24_put<M>(f24_row<M>(fdl, slot), k, v);
  else fdl[(size_t)slot * M + k] = v;
}
template <int SPEC, int M>
__device__ __forceinline__ float4 x_unit(const float2* fdl, int slot, int u) {
  if constexpr (SPEC == kSpecFP24) {
    float2 a, b;
    f24_unit<M>(f24_row<M>(fdl, slot), u, a, b);
    return make_float4(a.x, a.y, b.x, b.y);
  } else {
    return __ldg(reinterpret_cast<const float4*>(fdl) + (size_t)slot * (M / 2) + u);
  }
}

// ---------------------------------------------------------------------------
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_ir_kernel(EngChan* __restrict__ chans, const EngUpd* __restrict__ upd, const float2* __restrict__ tw) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  __shared__ float red[32];
  const int part = blockIdx.x;
  const EngUpd u = upd[blockIdx.y];
  const EngChan ch = chans[u.chan];
  if (part >= ch.P) return;
  // samples [part * M, part * M + M) of the row; zero at and after u.n
  const long long t0 = (long long)part * M;
  for (int n = threadIdx.x; n < M; n += T) {
    const long long t = t0 + 2 * n;
    float2 v = make_float2(0.f, 0.f);
    if (n < M / 2) {
      if (t < u.n) v.x = u.src[t];
      if (t + 1 < u.n) v.y = u.src[t + 1];
    }
    sm[n] = v;
  }
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
  if constexpr (kScaled<SPEC>) {
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
  if constexpr (SPEC == kSpecFP24) {
    void* row = f24_row<M>(ch.H, (size_t)u.slot * ch.P + part);
    for (int k = threadIdx.x; k < M; k += T) f24_put<M>(row, k, sm[k]);
  } else {
    for (int k = threadIdx.x; k < M; k += T)
      SpecT<SPEC>::put(ch.H, spec_index(ch, u.slot, part, M) + k, make_float2(sm[k].x * inv, sm[k].y * inv));
  }
}

// ---------------------------------------------------------------------------
// Two packed bins (one float4 of a delay-line row) per unit; spectra are float4
// (FP32) or uint2 (two half2 / bfloat162) per unit.
template <int SPEC, int M>
__device__ __forceinline__ void load_h2(const void* H, size_t idx2, float2& a, float2& b) {
  if constexpr (SPEC == kSpecFP24) {
    f24_unit<M>(f24_row<M>(H, idx2 / (M / 2)), (int)(idx2 % (M / 2)), a, b);
  } else if constexpr (SPEC == kSpecFP32) {
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

template <int SPEC, int M>
__device__ __forceinline__ float2 spec_bin(const EngChan& ch, int slot, int part, int k) {
  if constexpr (SPEC == kSpecFP24) {
    return f24_bin<M>(f24_row<M>(ch.H, (size_t)slot * ch.P + part), k);
  } else {
    float2 h = SpecT<SPEC>::get(ch.H, spec_index(ch, slot, part, M) + k);
    if constexpr (kScaled<SPEC>) {
      const float s = ch.scale[(size_t)slot * ch.P + part];
      h.x *= s;
      h.y *= s;
    }
    return h;
  }
}

// Partial-sum row of a channel: rows [2 parity][2 mode][nitem][M] float2; mode
// 0 = the IR in use for that block, 1 = a newly committed IR (swap block).
__device__ __forceinline__ float2* part_row(const EngChan& ch, int parity, int mode, int row, int M) {
  return ch.part + ((size_t)(parity * 2 + mode) * ch.nitem + row) * M;
}

// One work item: sum over partitions i in [w.i0, w.i1) of delay-line slot
// (ch.cur + i + fs_off) mod P times IR-spectrum partition i of `slot`, into
// part_row(parity, mode, w.row). M / 4 threads, units u and u + M / 4 each.
template <int LOG2M, int SPEC>
__device__ __forceinline__ void eng_item(const EngChan& ch, const EngItem& w, int slot, int fs_off, int parity,
                                         int mode) {
  constexpr int M = 1 << LOG2M, U = M / 2, T = M / 4, D = 2;
  const int P = ch.P;
  const size_t hb = ((size_t)slot * P * M) / 2;  // unit index of (slot, partition 0)
  const float* sc = kScaled<SPEC> ? ch.scale + (size_t)slot * P : nullptr;
  const int u0 = threadIdx.x, u1 = threadIdx.x + T;
  const bool dc = (u0 == 0);
  float2 a0 = make_float2(0.f, 0.f), a1 = a0, b0 = a0, b1 = a0;
  int fs = (ch.cur + w.i0 + fs_off) % P;
  int i = w.i0;
  for (; i + D <= w.i1; i += D) {
    float4 f0[D], f1[D];
    float2 p0[D], q0[D], p1[D], q1[D];
    float s[D];
#pragma unroll
    for (int q = 0; q < D; ++q) {
      f0[q] = x_unit<SPEC, M>(ch.fdl, fs, u0);
      f1[q] = x_unit<SPEC, M>(ch.fdl, fs, u1);
      const size_t hrow = hb + (size_t)(i + q) * U;
      load_h2<SPEC, M>(ch.H, hrow + u0, p0[q], q0[q]);
      load_h2<SPEC, M>(ch.H, hrow + u1, p1[q], q1[q]);
      s[q] = kScaled<SPEC> ? __ldg(sc + i + q) : 1.f;
      fs = (fs + 1 == P) ? 0 : fs + 1;
    }
#pragma unroll
    for (int q = 0; q < D; ++q) {
      if (kScaled<SPEC>) {
        p0[q].x *= s[q]; p0[q].y *= s[q]; q0[q].x *= s[q]; q0[q].y *= s[q];
        p1[q].x *= s[q]; p1[q].y *= s[q]; q1[q].x *= s[q]; q1[q].y *= s[q];
      }
      const float2 fa = make_float2(f0[q].x, f0[q].y), fb = make_float2(f0[q].z, f0[q].w);
      const float2 ga = make_float2(f1[q].x, f1[q].y), gb = make_float2(f1[q].z, f1[q].w);
      a0 = dc ? c_mac_dc(a0, fa, p0[q]) : c_mac(a0, fa, p0[q]);
      a1 = c_mac(a1, fb, q0[q]);
      b0 = c_mac(b0, ga, p1[q]);
      b1 = c_mac(b1, gb, q1[q]);
    }
  }
  for (; i < w.i1; ++i) {
    const float4 g0 = x_unit<SPEC, M>(ch.fdl, fs, u0), g1 = x_unit<SPEC, M>(ch.fdl, fs, u1);
    float2 pa, qa, pb, qb;
    const size_t hrow = hb + (size_t)i * U;
    load_h2<SPEC, M>(ch.H, hrow + u0, pa, qa);
    load_h2<SPEC, M>(ch.H, hrow + u1, pb, qb);
    if (kScaled<SPEC>) {
      const float s = __ldg(sc + i);
      pa.x *= s; pa.y *= s; qa.x *= s; qa.y *= s;
      pb.x *= s; pb.y *= s; qb.x *= s; qb.y *= s;
    }
    fs = (fs + 1 == P) ? 0 : fs + 1;
    const float2 fa = make_float2(g0.x, g0.y), fb = make_float2(g0.z, g0.w);
    const float2 ga = make_float2(g1.x, g1.y), gb = make_float2(g1.z, g1.w);
    a0 = dc ? c_mac_dc(a0, fa, pa) : c_mac(a0, fa, pa);
    a1 = c_mac(a1, fb, qa);
    b0 = c_mac(b0, ga, pb);
    b1 = c_mac(b1, gb, qb);
  }
  float4* dst = reinterpret_cast<float4*>(part_row(ch, parity, mode, w.row, M));
  dst[u0] = make_float4(a0.x, a0.y, a1.x, a1.y);
  dst[u1] = make_float4(b0.x, b0.y, b1.x, b1.y);
}

// Head of block k for one channel (state `ch` as at launch). Tail of the IR in
// use: the partial-sum rows of parity k plus X_{k-1} * H_1; on a swap block the
// same for the new IR (mode-1 rows), and the output crossfades.
template <int LOG2M, int SPEC>
__device__ __forceinline__ void eng_head(const EngChan& ch, float2* sm, const float* x, float* y,
                                         const float2* __restrict__ tw, int parity) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  float2* z = sm;
  float2* z2 = sm + M;
  const bool swap = ch.pending != 0;
  const int P = ch.P;
  const int cur = (ch.cur - 1 + P) % P;  // slot of X_k
  const int slot_old = ch.active, slot_new = 1 - ch.active;

  const bool x_vec = x && (reinterpret_cast<uintptr_t>(x) & 7) == 0;
  for (int n = threadIdx.x; n < M; n += T) {
    if (n < M / 2) {
      z[n] = reinterpret_cast<const float2*>(ch.prev)[n];
    } else if (!x) {
      z[n] = make_float2(0.f, 0.f);
    } else if (x_vec) {
      z[n] = reinterpret_cast<const float2*>(x)[n - M / 2];
    } else {
      const float* src = x + 2 * (n - M / 2);
      z[n] = make_float2(src[0], src[1]);
    }
  }
  __syncthreads();
  for (int n = threadIdx.x; n < M / 2; n += T) reinterpret_cast<float2*>(ch.prev)[n] = z[n + M / 2];
  fft_inplace<LOG2M, false>(z, tw);

  // X_k goes into delay-line slot cur; X_{k-1} (partition 1) is in ch.cur
  const float inv_n = 1.0f / (float)(2 * M);
  const float2* pa = part_row(ch, parity, 0, 0, M);
  const float2* pb = part_row(ch, parity, 1, 0, M);
  for (int k = threadIdx.x; k <= M / 2; k += T) {
    const int km = (k == 0) ? 0 : M - k;
    // tails: partial sums of the work items in item order, then partition 1
    float2 tk = make_float2(0.f, 0.f), tm = tk, uk = tk, um = tk;
    for (int r = 0; r < ch.nitem; ++r) {
      const float2 a = pa[(size_t)r * M + k], b = pa[(size_t)r * M + km];
      tk.x += a.x; tk.y += a.y;
      tm.x += b.x; tm.y += b.y;
      if (swap) {
        const float2 a1 = pb[(size_t)r * M + k], b1 = pb[(size_t)r * M + km];
        uk.x += a1.x; uk.y += a1.y;
        um.x += b1.x; um.y += b1.y;
      }
    }
    if (P > 1) {
      const float2 xk = x_bin<SPEC, M>(ch.fdl, ch.cur, k), xm = x_bin<SPEC, M>(ch.fdl, ch.cur, km);
      const float2 hk = spec_bin<SPEC, M>(ch, slot_old, 1, k);
      if (k == 0) {
        tk = c_mac_dc(tk, xk, hk);
        if (swap) uk = c_mac_dc(uk, xk, spec_bin<SPEC, M>(ch, slot_new, 1, 0));
      } else {
        tk = c_mac(tk, xk, hk);
        tm = c_mac(tm, xm, spec_bin<SPEC, M>(ch, slot_old, 1, km));
        if (swap) {
          uk = c_mac(uk, xk, spec_bin<SPEC, M>(ch, slot_new, 1, k));
          um = c_mac(um, xm, spec_bin<SPEC, M>(ch, slot_new, 1, km));
        }
      }
    }
    if (k == 0) {
      const float2 X = rfft_post_dc(z[0]);
      x_put<SPEC, M>(ch.fdl, cur, 0, X);
      z[0] = irfft_pre_dc(c_mac_dc(tk, X, spec_bin<SPEC, M>(ch, slot_old, 0, 0)), inv_n);
      if (swap) z2[0] = irfft_pre_dc(c_mac_dc(uk, X, spec_bin<SPEC, M>(ch, slot_new, 0, 0)), inv_n);
    } else {
      const float2 wk = __ldg(tw + k), wm = __ldg(tw + km);
      const float2 a = z[k], b = z[km];
      const float2 Xk = rfft_post(a, b, wk);
      const float2 Xm = rfft_post(b, a, wm);
      x_put<SPEC, M>(ch.fdl, cur, k, Xk);
      if (km != k) x_put<SPEC, M>(ch.fdl, cur, km, Xm);
      const float2 Ak = c_mac(tk, Xk, spec_bin<SPEC, M>(ch, slot_old, 0, k));
      const float2 Am = c_mac(tm, Xm, spec_bin<SPEC, M>(ch, slot_old, 0, km));
      z[k] = irfft_pre(Ak, Am, wk, inv_n);
      if (km != k) z[km] = irfft_pre(Am, Ak, wm, inv_n);
      if (swap) {
        const float2 Bk = c_mac(uk, Xk, spec_bin<SPEC, M>(ch, slot_new, 0, k));
        const float2 Bm = c_mac(um, Xm, spec_bin<SPEC, M>(ch, slot_new, 0, km));
        z2[k] = irfft_pre(Bk, Bm, wk, inv_n);
        if (km != k) z2[km] = irfft_pre(Bm, Bk, wm, inv_n);
      }
    }
  }
  __syncthreads();
  fft_inplace<LOG2M, true>(z, tw);
  if (swap) fft_inplace<LOG2M, true>(z2, tw);
  const float step = 1.0f / (float)M;
  const bool y_vec = (reinterpret_cast<uintptr_t>(y) & 7) == 0;
  for (int m = M / 2 + threadIdx.x; m < M; m += T) {
    const int i = 2 * (m - M / 2);
    float2 o = z[m];
    if (swap) {
      const float2 yn = z2[m];
      o = make_float2(yn.x * (step * (float)i) + o.x * (step * (float)(M - i)),
                      yn.y * (step * (float)(i + 1)) + o.y * (step * (float)(M - i - 1)));
    }
    if (y_vec) {
      reinterpret_cast<float2*>(y)[i / 2] = o;
    } else {
      y[i] = o.x;
      y[i + 1] = o.y;
    }
  }
}

template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_block_kernel(EngChan* __restrict__ chans, int nslots, const EngItem* __restrict__ items, int nitems,
                     const float* __restrict__ in_base, float* __restrict__ out_base, int ld,
                     const float2* __restrict__ tw, EngSync sync) {
  extern __shared__ float2 sm[];
  __shared__ int last;
  const long long k = *sync.block;  // blocks processed before this one
  const int parity = (int)(k & 1);
  // CTAs [0, stride) stream the work items and are dispatched first; the
  // heads follow and take the SM slots the item CTAs leave free, so heads and
  // items run side by side from the start of the launch.
  const int stride = (int)gridDim.x - nslots;
  if ((int)blockIdx.x >= stride) {
    const int c = (int)blockIdx.x - stride;
    const EngChan ch = chans[c];
    if (ch.run)
      eng_head<LOG2M, SPEC>(ch, sm, in_base ? in_base + (size_t)c * ld : nullptr, out_base + (size_t)c * ld, tw,
                            parity);
  } else {
    for (int it = (int)blockIdx.x; it < nitems; it += stride) {
      const EngItem w = items[it];
      if (w.chan < 0) continue;
      const EngChan ch = chans[w.chan];
      if (!ch.run) continue;
      // the next block's IR: the new one when this block swaps
      eng_item<LOG2M, SPEC>(ch, w, ch.pending ? 1 - ch.active : ch.active, -2, parity ^ 1, 0);
    }
  }
  // The last CTA to finish advances every channel and the block counter; every
  // CTA has read the state above before it counts itself done.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(sync.done, 1u) == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int c = threadIdx.x; c < nslots; c += blockDim.x) {
    EngChan* ch = chans + c;
    if (!ch->run) continue;
    ch->cur = (ch->cur - 1 + ch->P) % ch->P;
    if (ch->pending) {
      ch->active = 1 - ch->active;
      ch->pending = 0;
    }
  }
  if (threadIdx.x == 0) {
    *sync.block = k + 1;
    *sync.done = 0u;
  }
}

template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_commit_kernel(const EngChan* __restrict__ chans, const EngItem* __restrict__ items, int item0, int nitems,
                      const long long* __restrict__ block) {
  const int parity = (int)(*block & 1);  // the coming block
  for (int it = item0 + (int)blockIdx.x; it < item0 + nitems; it += gridDim.x) {
    const EngItem w = items[it];
    if (w.chan < 0) continue;
    const EngChan ch = chans[w.chan];
    if (!ch.pending) continue;
    eng_item<LOG2M, SPEC>(ch, w, 1 - ch.active, -1, parity, 1);
  }
}

// Marks channel slots [first, first + n) as holding a newly committed IR.
__global__ void eng_mark_pending_kernel(EngChan* __restrict__ chans, int first, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) chans[first + i].pending = 1;
}

template <int LOG2M, int SPEC>
cudaError_t attrs_t() {
  const int smem = 2 * (1 << LOG2M) * (int)sizeof(float2);
  cudaError_t e =
      cudaFuncSetAttribute(eng_block_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(eng_ir_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem / 2);
}

template <int LOG2M>
cudaError_t attrs_all() {
  cudaError_t e;
  if ((e = attrs_t<LOG2M, kSpecFP32>()) != cudaSuccess) return e;
  if ((e = attrs_t<LOG2M, kSpecFP16>()) != cudaSuccess) return e;
  if ((e = attrs_t<LOG2M, kSpecBF16>()) != cudaSuccess) return e;
  return attrs_t<LOG2M, kSpecFP24>();
}

template <int LOG2M, int SPEC>
cudaError_t ir_t(EngChan* chans, const EngUpd* upd, int nupd, int maxP, const float2* tw, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  dim3 grid(maxP, nupd);
  eng_ir_kernel<LOG2M, SPEC><<<grid, S::T, S::M * sizeof(float2), st>>>(chans, upd, tw);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t block_t(EngChan* chans, int nslots, const EngItem* items, int nitems, int tail_ctas, const float* in,
                    float* out, int ld, const float2* tw, EngSync sync, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_block_kernel<LOG2M, SPEC><<<nslots + tail_ctas, S::T, 2 * S::M * sizeof(float2), st>>>(
      chans, nslots, items, nitems, in, out, ld, tw, sync);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t commit_t(const EngChan* chans, const EngItem* items, int item0, int nitems, int grid,
                     const long long* block, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_commit_kernel<LOG2M, SPEC><<<grid, S::T, 0, st>>>(chans, items, item0, nitems, block);
  return cudaGetLastError();
}

#define ENG_DISPATCH(L2, SP, FN, ...)                                     \
  switch ((L2) * 4 + (SP)) {                                              \
    case 7 * 4 + 0: return FN<7, 0>(__VA_ARGS__);                         \
    case 7 * 4 + 1: return FN<7, 1>(__VA_ARGS__);                         \
    case 7 * 4 + 2: return FN<7, 2>(__VA_ARGS__);                         \
    case 7 * 4 + 3: return FN<7, 3>(__VA_ARGS__);                         \
    case 8 * 4 + 0: return FN<8, 0>(__VA_ARGS__);                         \
    case 8 * 4 + 1: return FN<8, 1>(__VA_ARGS__);                         \
    case 8 * 4 + 2: return FN<8, 2>(__VA_ARGS__);                         \
    case 8 * 4 + 3: return FN<8, 3>(__VA_ARGS__);                         \
    case 9 * 4 + 0: return FN<9, 0>(__VA_ARGS__);                         \
    case 9 * 4 + 1: return FN<9, 1>(__VA_ARGS__);                         \
    case 9 * 4 + 2: return FN<9, 2>(__VA_ARGS__);                         \
    case 9 * 4 + 3: return FN<9, 3>(__VA_ARGS__);                         \
    case 10 * 4 + 0: return FN<10, 0>(__VA_ARGS__);                       \
    case 10 * 4 + 1: return FN<10, 1>(__VA_ARGS__);                       \
    case 10 * 4 + 2: return FN<10, 2>(__VA_ARGS__);                       \
    case 10 * 4 + 3: return FN<10, 3>(__VA_ARGS__);                       \
    case 11 * 4 + 0: return FN<11, 0>(__VA_ARGS__);                       \
    case 11 * 4 + 1: return FN<11, 1>(__VA_ARGS__);                       \
    case 11 * 4 + 2: return FN<11, 2>(__VA_ARGS__);                       \
    case 11 * 4 + 3: return FN<11, 3>(__VA_ARGS__);                       \
    default: return cudaErrorInvalidValue;                                \
  }

}  // namespace

cudaError_t eng_prepare() {
  static OncePerDevice once;
  return once.run([] {
    cudaError_t e;
    if ((e = attrs_all<7>()) != cudaSuccess) return e;
    if ((e = attrs_all<8>()) != cudaSuccess) return e;
    if ((e = attrs_all<9>()) != cudaSuccess) return e;
    if ((e = attrs_all<10>()) != cudaSuccess) return e;
    return attrs_all<11>();
  });
}

cudaError_t eng_launch_ir(int log2B, int spec, EngChan* chans, const EngUpd* upd, int nupd, int maxP,
                          const float2* tw, cudaStream_t st) {
  if (nupd <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, ir_t, chans, upd, nupd, maxP, tw, st);
}

cudaError_t eng_launch_block(int log2B, int spec, EngChan* chans, int nslots, const EngItem* items, int nitems,
                             int tail_ctas, const float* in, float* out, int ld, const float2* tw, EngSync sync,
                             cudaStream_t st) {
  if (nslots <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, block_t, chans, nslots, items, nitems, tail_ctas, in, out, ld, tw, sync, st);
}

cudaError_t eng_launch_mark_pending(EngChan* chans, int first, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  eng_mark_pending_kernel<<<(n + 255) / 256, 256, 0, st>>>(chans, first, n);
  return cudaGetLastError();
}

cudaError_t eng_launch_commit(int log2B, int spec, const EngChan* chans, const EngItem* items, int item0,
                              int nitems, int grid, const long long* block, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, commit_t, chans, items, item0, nitems, grid, block, st);
}

}  // namespace tanb
