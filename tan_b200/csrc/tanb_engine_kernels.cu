// Kernels of the batched engine: every channel of every open session runs in
// ONE graph launch per audio block.
//
//   eng_ir_kernel      one CTA per (IR partition, updated channel): R2C of the
//                      partition, optional FP16/BF16 quantisation with a
//                      power-of-two per-partition scale, stored in the idle slot
//                      (runs on the engine's update stream); eng_level_ir_kernel
//                      the same for the partitions of a non-uniform level
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
//                      Work items of non-uniform levels (one bin slice of the
//                      level's partitions per base block, so that a level's tail
//                      is spread over the p base blocks of its period) run in
//                      the same grid.
//   eng_level_head_kernel  beside the block kernel, in the same graph, at the
//                      blocks where a level of that size completes: one CTA per
//                      level record, R2C of the level's 2N frame (input history
//                      plus this block's input row), insert into the level's
//                      delay line, partitions 0 and 1 plus the partial rows,
//                      C2R, the N outputs into the level's output ring at their
//                      delayed position. It reads no data the block kernel
//                      writes in this block and counts into the same
//                      completion counter.
//   eng_commit_kernel  partial sums of a newly committed IR for the coming block
//                      (before that block's launch), from the current delay line;
//                      eng_level_commit_* the same for non-uniform levels: the
//                      partial rows of the level blocks still to come and the
//                      output of level blocks whose output is still to be
//                      played, recomputed with the new IR
//
// The per-block sums are the reference's head and tail
// (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:2380-2643);
// the batching across channels with a channel map is the role the reference's
// GPU engine gives processAccum (tan/tanlibrary/src/Graal/GraalConv.cpp:1883-2145);
// the non-uniform levels are the multiple-block partitions of the reference's
// CPU non-uniform method (ConvolutionImpl.cpp:224-246, 2416-2428) generalised
// to a ladder of sizes, each spread over its period as that method spreads its
// tail over M blocks.
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

// The same for rows whose length n is known only at run time (level rows).
__device__ __forceinline__ void f24_unit_rt(const void* row, int n, int u, float2& a, float2& b) {
  const uint2 hi = __ldg(reinterpret_cast<const uint2*>(row) + u);
  const unsigned lo = __ldg(reinterpret_cast<const unsigned*>(static_cast<const char*>(row) + 4 * (size_t)n) + u);
  a = make_float2(f24_decode(hi.x & 0xFFFFu, lo & 0xFFu), f24_decode(hi.x >> 16, (lo >> 8) & 0xFFu));
  b = make_float2(f24_decode(hi.y & 0xFFFFu, (lo >> 16) & 0xFFu), f24_decode(hi.y >> 16, lo >> 24));
}
__device__ __forceinline__ const void* f24_row_rt(const void* base, size_t row, int n) {
  return static_cast<const char*>(base) + row * (size_t)(6 * (size_t)n);
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
// R2C of one IR partition into IR slot `slot` of a spectrum table [2][P][M]
// (with scales [2][P] for FP16 / BF16): samples [t0, t0 + M) of `src`, zero at
// and after n, zero-padded to 2M. Every thread of the CTA calls it.
template <int LOG2M, int SPEC>
__device__ __forceinline__ void ir_partition(void* H, float* scale_tab, int P, int slot, int part, const float* src,
                                             long long t0, long long n, const float2* __restrict__ tw, float2* sm) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  __shared__ float red[32];
  for (int q = threadIdx.x; q < M; q += T) {
    const long long t = t0 + 2 * q;
    float2 v = make_float2(0.f, 0.f);
    if (q < M / 2) {
      if (t < n) v.x = src[t];
      if (t + 1 < n) v.y = src[t + 1];
    }
    sm[q] = v;
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
    // a partition of denormal samples: keep the scale a normal number (2^-149
    // would round to zero and its inverse overflow)
    e = e < -126 ? -126 : e;
    scale = ldexpf(1.0f, e);
    if (threadIdx.x == 0) scale_tab[(size_t)slot * P + part] = scale;
  }
  const float inv = 1.0f / scale;  // exact: power of two
  const size_t row = (size_t)slot * P + part;
  if constexpr (SPEC == kSpecFP24) {
    void* r = f24_row<M>(H, row);
    for (int k = threadIdx.x; k < M; k += T) f24_put<M>(r, k, sm[k]);
  } else {
    for (int k = threadIdx.x; k < M; k += T)
      SpecT<SPEC>::put(H, row * M + k, make_float2(sm[k].x * inv, sm[k].y * inv));
  }
}

template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_ir_kernel(EngChan* __restrict__ chans, const EngUpd* __restrict__ upd, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const int part = blockIdx.x;
  const EngUpd u = upd[blockIdx.y];
  const EngChan ch = chans[u.chan];
  if (part >= ch.P) return;
  ir_partition<LOG2M, SPEC>(ch.H, ch.scale, ch.P, u.slot, part, u.src, (long long)part * (1 << LOG2M), u.n, tw, sm);
}

// Partitions of non-uniform levels of one size (2^LOG2M): partition `part` of
// level record u.lvl covers taps [off + part M, off + (part + 1) M).
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_level_ir_kernel(EngLevel* __restrict__ levels, const EngLvlUpd* __restrict__ upd,
                        const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const int part = blockIdx.x;
  const EngLvlUpd u = upd[blockIdx.y];
  const EngLevel lv = levels[u.lvl];
  if (part >= lv.K) return;
  ir_partition<LOG2M, SPEC>(lv.H, lv.scale, lv.K, u.slot, part, u.src, lv.off + (long long)part * (1 << LOG2M), u.n,
                            tw, sm);
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

// spec_bin with the partition's scale already loaded (`sc`, FP16 / BF16 only):
// the same value, for loops that read many bins of one partition.
template <int SPEC, int M>
__device__ __forceinline__ float2 spec_bin_sc(const EngChan& ch, int slot, int part, int k, float sc) {
  if constexpr (kScaled<SPEC>) {
    float2 h = SpecT<SPEC>::get(ch.H, spec_index(ch, slot, part, M) + k);
    h.x *= sc;
    h.y *= sc;
    return h;
  } else {
    return spec_bin<SPEC, M>(ch, slot, part, k);
  }
}

// Scale of IR partition `part` of `slot` (1 for unscaled spectra).
template <int SPEC>
__device__ __forceinline__ float spec_scale(const EngChan& ch, int slot, int part) {
  if constexpr (kScaled<SPEC>) return ch.scale[(size_t)slot * ch.P + part];
  else return 1.f;
}

// Partial-sum row of a channel: rows [2 parity][2 mode][nitem][M] float2; mode
// 0 = the IR in use for that block, 1 = a newly committed IR (swap block).
__device__ __forceinline__ float2* part_row(const EngChan& ch, int parity, int mode, int row, int M) {
  return ch.part + ((size_t)(parity * 2 + mode) * ch.nitem + row) * M;
}

// One work item: sum over partitions i in [w.i0, w.i1) of delay-line slot
// (ch.cur + i + fs_off) mod P times IR-spectrum partition i of `slot`, into
// part_row(parity, mode, w.row), over half w.slice of the row's bins: M / 4
// threads, one float4 unit (two bins) each, four partitions' loads in flight
// (a base item covers half the bins, so the latency chain of one item is half
// as long and a channel's two halves run as two items).
template <int LOG2M, int SPEC>
__device__ __forceinline__ void eng_item(const EngChan& ch, const EngItem& w, int slot, int fs_off, int parity,
                                         int mode) {
  constexpr int M = 1 << LOG2M, U = M / 2, T = M / 4, D = 4;
  const int P = ch.P;
  const size_t hb = ((size_t)slot * P * M) / 2;  // unit index of (slot, partition 0)
  const float* sc = kScaled<SPEC> ? ch.scale + (size_t)slot * P : nullptr;
  const int u = w.slice * T + threadIdx.x;
  const bool dc = (u == 0);
  float2 a0 = make_float2(0.f, 0.f), a1 = a0;
  int fs = (ch.cur + w.i0 + fs_off) % P;
  int i = w.i0;
  for (; i + D <= w.i1; i += D) {
    float4 f[D];
    float2 p[D], q[D];
    float s[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      f[j] = x_unit<SPEC, M>(ch.fdl, fs, u);
      load_h2<SPEC, M>(ch.H, hb + (size_t)(i + j) * U + u, p[j], q[j]);
      s[j] = kScaled<SPEC> ? __ldg(sc + i + j) : 1.f;
      fs = (fs + 1 == P) ? 0 : fs + 1;
    }
#pragma unroll
    for (int j = 0; j < D; ++j) {
      if (kScaled<SPEC>) {
        p[j].x *= s[j]; p[j].y *= s[j]; q[j].x *= s[j]; q[j].y *= s[j];
      }
      const float2 fa = make_float2(f[j].x, f[j].y), fb = make_float2(f[j].z, f[j].w);
      a0 = dc ? c_mac_dc(a0, fa, p[j]) : c_mac(a0, fa, p[j]);
      a1 = c_mac(a1, fb, q[j]);
    }
  }
  for (; i < w.i1; ++i) {
    const float4 g = x_unit<SPEC, M>(ch.fdl, fs, u);
    float2 pa, qa;
    load_h2<SPEC, M>(ch.H, hb + (size_t)i * U + u, pa, qa);
    if (kScaled<SPEC>) {
      const float s = __ldg(sc + i);
      pa.x *= s; pa.y *= s; qa.x *= s; qa.y *= s;
    }
    fs = (fs + 1 == P) ? 0 : fs + 1;
    a0 = dc ? c_mac_dc(a0, make_float2(g.x, g.y), pa) : c_mac(a0, make_float2(g.x, g.y), pa);
    a1 = c_mac(a1, make_float2(g.z, g.w), qa);
  }
  reinterpret_cast<float4*>(part_row(ch, parity, mode, w.row, M))[u] = make_float4(a0.x, a0.y, a1.x, a1.y);
}

// ---------------------------------------------------------------------------
// Non-uniform levels. Rows of N bins (N known at run time in the work items,
// at compile time in the level heads).

// Delay-line slot of level block j (any sign): Kr-1 - (j mod Kr). Slots of
// negative blocks are never written and hold zeros.
__device__ __forceinline__ int lv_slot(long long j, int Kr) {
  long long m = j % Kr;
  if (m < 0) m += Kr;
  return Kr - 1 - (int)m;
}

// float4 unit u (bins 2u, 2u + 1) of delay-line slot `slot` of a level.
template <int SPEC>
__device__ __forceinline__ float4 lv_x_unit(const float2* fdl, int n, int slot, int u) {
  if constexpr (SPEC == kSpecFP24) {
    float2 a, b;
    f24_unit_rt(f24_row_rt(fdl, slot, n), n, u, a, b);
    return make_float4(a.x, a.y, b.x, b.y);
  } else {
    return __ldg(reinterpret_cast<const float4*>(fdl) + (size_t)slot * (n / 2) + u);
  }
}

// Bins 2u, 2u + 1 of spectrum row `row` (= slot * K + partition) of a level,
// unscaled.
template <int SPEC>
__device__ __forceinline__ void lv_h2(const void* H, int n, size_t row, int u, float2& a, float2& b) {
  if constexpr (SPEC == kSpecFP24) {
    f24_unit_rt(f24_row_rt(H, row, n), n, u, a, b);
  } else if constexpr (SPEC == kSpecFP32) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(H) + row * (n / 2) + u);
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
  } else {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(H) + row * (n / 2) + u);
    if constexpr (SPEC == kSpecFP16) {
      a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
      b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    } else {
      a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
      b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
    }
  }
}

// Bin k of spectrum partition `part` of IR slot `slot` of a level of M bins
// (scaled).
template <int SPEC, int M>
__device__ __forceinline__ float2 lv_spec_bin(const EngLevel& lv, int slot, int part, int k) {
  const size_t row = (size_t)slot * lv.K + part;
  if constexpr (SPEC == kSpecFP24) {
    return f24_bin<M>(f24_row<M>(lv.H, row), k);
  } else {
    float2 h = SpecT<SPEC>::get(lv.H, row * M + k);
    if constexpr (kScaled<SPEC>) {
      const float s = lv.scale[row];
      h.x *= s;
      h.y *= s;
    }
    return h;
  }
}

// One level work item for level block jb: sum over partitions i in
// [w.i0, w.i1) of X_{jb - i} times IR partition i of `slot`, over the bins of
// slice `slice` (B bins: units [slice B / 2, (slice + 1) B / 2)), into partial
// row w.row of parity jb & 1. B / 4 threads, two units each, as eng_item.
template <int LOG2B, int SPEC>
__device__ __noinline__ void eng_level_item(const EngLevel& lv, const EngItem& w, int slot, long long jb, int slice) {
  constexpr int Bn = 1 << LOG2B, T = Bn / 4, D = 2;
  const int n = 1 << lv.log2N, K = lv.K, Kr = lv.Kr;
  const int u0 = slice * (Bn / 2) + threadIdx.x, u1 = u0 + T;
  const bool dc = (u0 == 0);
  const float* sc = kScaled<SPEC> ? lv.scale + (size_t)slot * K : nullptr;
  float2 a0 = make_float2(0.f, 0.f), a1 = a0, b0 = a0, b1 = a0;
  int fs = lv_slot(jb - w.i0, Kr);
  int i = w.i0;
  for (; i + D <= w.i1; i += D) {
    float4 f0[D], f1[D];
    float2 p0[D], q0[D], p1[D], q1[D];
    float s[D];
#pragma unroll
    for (int q = 0; q < D; ++q) {
      f0[q] = lv_x_unit<SPEC>(lv.fdl, n, fs, u0);
      f1[q] = lv_x_unit<SPEC>(lv.fdl, n, fs, u1);
      const size_t row = (size_t)slot * K + i + q;
      lv_h2<SPEC>(lv.H, n, row, u0, p0[q], q0[q]);
      lv_h2<SPEC>(lv.H, n, row, u1, p1[q], q1[q]);
      s[q] = kScaled<SPEC> ? __ldg(sc + i + q) : 1.f;
      fs = (fs + 1 == Kr) ? 0 : fs + 1;
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
    const float4 g0 = lv_x_unit<SPEC>(lv.fdl, n, fs, u0), g1 = lv_x_unit<SPEC>(lv.fdl, n, fs, u1);
    float2 pa, qa, pb, qb;
    const size_t row = (size_t)slot * K + i;
    lv_h2<SPEC>(lv.H, n, row, u0, pa, qa);
    lv_h2<SPEC>(lv.H, n, row, u1, pb, qb);
    if (kScaled<SPEC>) {
      const float s = __ldg(sc + i);
      pa.x *= s; pa.y *= s; qa.x *= s; qa.y *= s;
      pb.x *= s; pb.y *= s; qb.x *= s; qb.y *= s;
    }
    fs = (fs + 1 == Kr) ? 0 : fs + 1;
    const float2 fa = make_float2(g0.x, g0.y), fb = make_float2(g0.z, g0.w);
    const float2 ga = make_float2(g1.x, g1.y), gb = make_float2(g1.z, g1.w);
    a0 = dc ? c_mac_dc(a0, fa, pa) : c_mac(a0, fa, pa);
    a1 = c_mac(a1, fb, qa);
    b0 = c_mac(b0, ga, pb);
    b1 = c_mac(b1, gb, qb);
  }
  float4* dst = reinterpret_cast<float4*>(lv.part + ((size_t)((jb & 1) * lv.ngroup + w.row)) * n);
  dst[u0] = make_float4(a0.x, a0.y, a1.x, a1.y);
  dst[u1] = make_float4(b0.x, b0.y, b1.x, b1.y);
}

__device__ __forceinline__ const float* row_in(const EngRows& r, int c) {
  return r.in_tab ? r.in_tab[c] : (r.in_base ? r.in_base + (size_t)c * r.ld : nullptr);
}
__device__ __forceinline__ float* row_out(const EngRows& r, int c) {
  return r.out_tab ? r.out_tab[c] : (r.out_base ? r.out_base + (size_t)c * r.ld : nullptr);
}

// Head of block k for one channel (state `ch` as at launch). Tail of the IR in
// use: the partial-sum rows of parity k plus X_{k-1} * H_1; on a swap block the
// same for the new IR (mode-1 rows), and the output crossfades. A non-uniform
// channel also appends x_k to its input history and adds its levels' output
// rings (of the IR slot in use; on a swap block those of each IR to its side
// of the crossfade) in level order.
//
// The head shares the GPU with the launch's item CTAs, which keep HBM busy
// and stream through L1, so each dependent round trip to memory costs
// microseconds. Every load of the head is therefore issued before the forward
// transform: the frame to registers, and the tails (partial-sum rows,
// X_{k-1} * H_1) and H_0 reduced and parked in shared memory (st, sh; on a
// swap block the new IR's tail in z2, which the bin loop reads before it
// overwrites it). Each thread reads back only the bins it wrote. The
// operations and their order are those of a single bin loop.
// With `tw_stage` the twiddle table also goes to shared memory, by
// asynchronous copies (no registers held): for launches of few heads, whose
// transforms would otherwise wait on L2 at every stage. Launches of many
// heads read it from global memory, where the heads on one SM share it in
// L1 and the item CTAs keep the L1 capacity for their loads in flight.
template <int LOG2M, int SPEC>
__device__ __forceinline__ void eng_head(const EngChan& ch, float2* sm, const float* x, float* y,
                                         const float2* __restrict__ twg, bool tw_stage, long long kblk) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T, E = S::E;
  const int parity = (int)(kblk & 1);
  float2* z = sm;
  float2* z2 = sm + M;
  float2* st = sm + 2 * M;  // tail of the IR in use, per bin
  float2* sh = sm + 3 * M;  // H_0 of the IR in use, per bin
  // twiddles W_2M^j, j < 3M/2 (all the transforms read)
  const float2* tw = twg;
  if (tw_stage) {
    float2* tws = sm + 4 * M;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int i = threadIdx.x + e * T;  // float4 i of 3M/4
      const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(reinterpret_cast<float4*>(tws) + i));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                   "l"(reinterpret_cast<const float4*>(twg) + i)
                   : "memory");
    }
    tw = tws;
  }
  const bool swap = ch.pending != 0;
  const int P = ch.P;
  const int cur = (ch.cur - 1 + P) % P;  // slot of X_k
  const int slot_old = ch.active, slot_new = 1 - ch.active;

  // what the level rings' pass after the inverse transforms needs, kept in
  // shared memory rather than in registers across the transforms
  __shared__ long long s_t0;
  __shared__ int s_slot_old;
  __shared__ const EngNu* s_nu;
  if (threadIdx.x == 0) {
    s_t0 = kblk * M;
    s_slot_old = slot_old;
    s_nu = ch.nu;
  }
  const bool x_vec = x && (reinterpret_cast<uintptr_t>(x) & 7) == 0;
  float2 zr[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int n = threadIdx.x + e * T;
    if (n < M / 2) {
      zr[e] = reinterpret_cast<const float2*>(ch.prev)[n];
    } else if (!x) {
      zr[e] = make_float2(0.f, 0.f);
    } else if (x_vec) {
      zr[e] = reinterpret_cast<const float2*>(x)[n - M / 2];
    } else {
      const float* src = x + 2 * (n - M / 2);
      zr[e] = make_float2(src[0], src[1]);
    }
  }
  // tails: partial sums of the work items in item order, then partition 1;
  // and partition 0 for the product with X_k. Bins k and M - k per thread,
  // k < M/2, with bin M/2 beside bin 0 (both use one bin of the pair alone):
  // two pairs for each of the M/4 threads.
  constexpr int KQ = (M / 2) / T;
  static_assert(KQ * T == M / 2, "the head runs M/4 threads");
  const float2* pa = part_row(ch, parity, 0, 0, M);
  const float sc0 = spec_scale<SPEC>(ch, slot_old, 0), sc1 = P > 1 ? spec_scale<SPEC>(ch, slot_old, 1) : 1.f;
#pragma unroll
  for (int q = 0; q < KQ; ++q) {
    const int k = threadIdx.x + q * T;
    const int km = (k == 0) ? M / 2 : M - k;
    float2 tk = make_float2(0.f, 0.f), tm = tk;
#pragma unroll 4
    for (int r = 0; r < ch.nitem; ++r) {
      const float2 a = pa[(size_t)r * M + k], b = pa[(size_t)r * M + km];
      tk.x += a.x; tk.y += a.y;
      tm.x += b.x; tm.y += b.y;
    }
    const float2 h0k = spec_bin_sc<SPEC, M>(ch, slot_old, 0, k, sc0);
    const float2 h0m = spec_bin_sc<SPEC, M>(ch, slot_old, 0, km, sc0);
    if (P > 1) {
      const float2 xk = x_bin<SPEC, M>(ch.fdl, ch.cur, k), xm = x_bin<SPEC, M>(ch.fdl, ch.cur, km);
      const float2 h1k = spec_bin_sc<SPEC, M>(ch, slot_old, 1, k, sc1);
      tk = (k == 0) ? c_mac_dc(tk, xk, h1k) : c_mac(tk, xk, h1k);
      tm = c_mac(tm, xm, spec_bin_sc<SPEC, M>(ch, slot_old, 1, km, sc1));
    }
    st[k] = tk;
    st[km] = tm;
    sh[k] = h0k;
    sh[km] = h0m;
  }
  if (swap) {
    // the same for the new IR, into z2
    const float2* pb = part_row(ch, parity, 1, 0, M);
    for (int q = 0; q < KQ; ++q) {
      const int k = threadIdx.x + q * T;
      const int km = (k == 0) ? M / 2 : M - k;
      float2 uk = make_float2(0.f, 0.f), um = uk;
      for (int r = 0; r < ch.nitem; ++r) {
        const float2 a1 = pb[(size_t)r * M + k], b1 = pb[(size_t)r * M + km];
        uk.x += a1.x; uk.y += a1.y;
        um.x += b1.x; um.y += b1.y;
      }
      if (P > 1) {
        const float2 xk = x_bin<SPEC, M>(ch.fdl, ch.cur, k), xm = x_bin<SPEC, M>(ch.fdl, ch.cur, km);
        uk = (k == 0) ? c_mac_dc(uk, xk, spec_bin<SPEC, M>(ch, slot_new, 1, 0))
                      : c_mac(uk, xk, spec_bin<SPEC, M>(ch, slot_new, 1, k));
        um = c_mac(um, xm, spec_bin<SPEC, M>(ch, slot_new, 1, km));
      }
      z2[k] = uk;
      z2[km] = um;
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) z[threadIdx.x + e * T] = zr[e];
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  for (int n = threadIdx.x; n < M / 2; n += T) reinterpret_cast<float2*>(ch.prev)[n] = z[n + M / 2];
  if (ch.nu) {
    // the level heads of later blocks read this block's samples from here
    const EngNu* nu = ch.nu;
    float* ring = nu->in_ring;
    const long long t0 = kblk * M;
    const int mask = nu->rin - 1;
    for (int n = threadIdx.x; n < M / 2; n += T) {
      const float2 v = z[n + M / 2];
      ring[(t0 + 2 * n) & mask] = v.x;
      ring[(t0 + 2 * n + 1) & mask] = v.y;
    }
  }
  fft_inplace<LOG2M, false>(z, tw);

  // X_k goes into delay-line slot cur; X_{k-1} (partition 1) is in ch.cur
  const float inv_n = 1.0f / (float)(2 * M);
  for (int k = threadIdx.x; k <= M / 2; k += T) {
    const int km = (k == 0) ? 0 : M - k;
    const float2 tk = st[k], tm = st[km];
    // the new IR's tail and H_0 on a swap block
    float2 uk = make_float2(0.f, 0.f), um = uk, gk = uk, gm = uk;
    if (swap) {
      uk = z2[k];
      um = z2[km];
      gk = spec_bin<SPEC, M>(ch, slot_new, 0, k);
      gm = spec_bin<SPEC, M>(ch, slot_new, 0, km);
    }
    if (k == 0) {
      const float2 X = rfft_post_dc(z[0]);
      x_put<SPEC, M>(ch.fdl, cur, 0, X);
      z[0] = irfft_pre_dc(c_mac_dc(tk, X, sh[0]), inv_n);
      if (swap) z2[0] = irfft_pre_dc(c_mac_dc(uk, X, gk), inv_n);
    } else {
      const float2 wk = tw[k], wm = tw[km];
      const float2 a = z[k], b = z[km];
      const float2 Xk = rfft_post(a, b, wk);
      const float2 Xm = rfft_post(b, a, wm);
      x_put<SPEC, M>(ch.fdl, cur, k, Xk);
      if (km != k) x_put<SPEC, M>(ch.fdl, cur, km, Xm);
      const float2 Ak = c_mac(tk, Xk, sh[k]);
      const float2 Am = c_mac(tm, Xm, sh[km]);
      z[k] = irfft_pre(Ak, Am, wk, inv_n);
      if (km != k) z[km] = irfft_pre(Am, Ak, wm, inv_n);
      if (swap) {
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
  if (!y) return;
  if (const EngNu* nu = s_nu) {
    // the levels' outputs for this block, added in level order to each IR's
    // result (each thread updates the entries it writes out below)
    const long long t0 = s_t0;
    const int so = s_slot_old;
#pragma unroll 1
    for (int l = 0; l < nu->nlv; ++l) {
      const int mask = nu->R[l] - 1;
      const float* ro = nu->ring[l] + (size_t)so * nu->R[l];
      const float* rn = nu->ring[l] + (size_t)(1 - so) * nu->R[l];
#pragma unroll 1
      for (int m = M / 2 + threadIdx.x; m < M; m += T) {
        const long long t = t0 + 2 * (m - M / 2);
        z[m].x += ro[t & mask];
        z[m].y += ro[(t + 1) & mask];
        if (swap) {
          z2[m].x += rn[t & mask];
          z2[m].y += rn[(t + 1) & mask];
        }
      }
    }
  }
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

// Every CTA of a block (block kernel and level heads alike) counts itself once
// it has read the channel state; the last of `total` advances every channel
// slot and the block counter.
__device__ __forceinline__ void finish_block(EngChan* __restrict__ chans, int nslots, EngSync sync, unsigned total,
                                             long long k) {
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(sync.done, 1u) == total - 1) ? 1 : 0;
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

// At most 64 registers per thread: the launch's item CTAs and heads share the
// SMs, 1024 threads each (tail_ctas in the host code counts on it).
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T, 1024 / FftShape<LOG2M>::T)
    eng_block_kernel(EngChan* __restrict__ chans, int nslots, const EngItem* __restrict__ items, int nitems,
                     const EngLevel* __restrict__ levels, EngRows rows, const float2* __restrict__ tw, int tw_stage,
                     EngSync sync, unsigned total) {
  extern __shared__ __align__(16) float2 sm[];  // 16-byte copies into the head's twiddle table
  const long long k = *sync.block;  // blocks processed before this one
  const int parity = (int)(k & 1);
  // CTAs [0, stride) stream the work items and are dispatched first; the
  // heads follow and take the SM slots the item CTAs leave free, so heads and
  // items run side by side from the start of the launch.
  const int stride = (int)gridDim.x - nslots;
  if ((int)blockIdx.x >= stride) {
    const int c = (int)blockIdx.x - stride;
    const EngChan ch = chans[c];
    if (ch.run) eng_head<LOG2M, SPEC>(ch, sm, row_in(rows, c), row_out(rows, c), tw, tw_stage != 0, k);
  } else {
    for (int it = (int)blockIdx.x; it < nitems; it += stride) {
      const EngItem w = items[it];
      if (w.chan < 0) continue;
      const EngChan ch = chans[w.chan];
      if (!ch.run) continue;
      // the next block's IR: the new one when this block swaps
      const int slot = ch.pending ? 1 - ch.active : ch.active;
      if (w.lvl < 0) {
        eng_item<LOG2M, SPEC>(ch, w, slot, -2, parity ^ 1, 0);
      } else {
        // level block floor(k / p) + 1, its slice k mod p
        const EngLevel lv = levels[w.lvl];
        const int pshift = lv.log2N - LOG2M;
        eng_level_item<LOG2M, SPEC>(lv, w, slot, (k >> pshift) + 1, (int)(k & ((1LL << pshift) - 1)));
      }
    }
  }
  finish_block(chans, nslots, sync, total, k);
}

// Head of level block j = (k + 1) / p - 1 of every level record of one size
// class (2^LOG2M) at a block k where that size is due: frame = input samples
// [(j-1) N, (j+1) N) (the last B of them, this block's, from the input row),
// X_j into the level's delay line, Y = sum of the partial rows (parity j & 1,
// in row order) + X_{j-1} H_1 + X_j H_0, C2R, samples [N, 2N) of the result
// into the output ring of the IR in effect after this block at positions
// off + jN + i. It reads no data the block kernel of this block writes.
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_level_head_kernel(EngChan* __restrict__ chans, int nslots, const EngLevel* __restrict__ levels, int log2B,
                          EngRows rows, const float2* __restrict__ tw, EngSync sync, unsigned total) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  const long long k = *sync.block;
  const EngLevel lv = levels[blockIdx.x];
  const int pshift = LOG2M - log2B;
  bool work = lv.chan >= 0 && ((k + 1) & ((1LL << pshift) - 1)) == 0;
  EngChan ch{};
  if (work) {
    ch = chans[lv.chan];
    work = ch.run != 0;
  }
  if (work) {
    const long long j = ((k + 1) >> pshift) - 1;
    const int slot = ch.pending ? 1 - ch.active : ch.active;
    const EngNu* nu = ch.nu;
    const float* hist = nu->in_ring;
    const int hmask = nu->rin - 1;
    const float* x = row_in(rows, lv.chan);
    const long long s0 = (j - 1) * M, kB = k << log2B;
    float2* z = sm;
    for (int n = threadIdx.x; n < M; n += T) {
      const long long a = s0 + 2 * n;  // even, and kB is even: a and a + 1 on one side
      float2 v = make_float2(0.f, 0.f);
      if (a >= 0 && a < kB) {
        v = make_float2(hist[a & hmask], hist[(a + 1) & hmask]);
      } else if (a >= kB && x) {
        v = make_float2(x[a - kB], x[a + 1 - kB]);
      }
      z[n] = v;
    }
    __syncthreads();
    fft_inplace<LOG2M, false>(z, tw);
    const int K = lv.K, Kr = lv.Kr;
    const int cur = lv_slot(j, Kr), prv = lv_slot(j - 1, Kr);
    const float2* prow = lv.part + (size_t)((j & 1) * lv.ngroup) * M;
    const float inv_n = 1.0f / (float)(2 * M);
    for (int kk = threadIdx.x; kk <= M / 2; kk += T) {
      const int km = (kk == 0) ? 0 : M - kk;
      float2 tk = make_float2(0.f, 0.f), tm = tk;
      for (int r = 0; r < lv.ngroup; ++r) {
        const float2 a = prow[(size_t)r * M + kk], b = prow[(size_t)r * M + km];
        tk.x += a.x; tk.y += a.y;
        tm.x += b.x; tm.y += b.y;
      }
      if (K > 1) {
        const float2 xk = x_bin<SPEC, M>(lv.fdl, prv, kk), xm = x_bin<SPEC, M>(lv.fdl, prv, km);
        if (kk == 0) {
          tk = c_mac_dc(tk, xk, lv_spec_bin<SPEC, M>(lv, slot, 1, 0));
        } else {
          tk = c_mac(tk, xk, lv_spec_bin<SPEC, M>(lv, slot, 1, kk));
          tm = c_mac(tm, xm, lv_spec_bin<SPEC, M>(lv, slot, 1, km));
        }
      }
      if (kk == 0) {
        const float2 X = rfft_post_dc(z[0]);
        x_put<SPEC, M>(lv.fdl, cur, 0, X);
        z[0] = irfft_pre_dc(c_mac_dc(tk, X, lv_spec_bin<SPEC, M>(lv, slot, 0, 0)), inv_n);
      } else {
        const float2 wk = __ldg(tw + kk), wm = __ldg(tw + km);
        const float2 a = z[kk], b = z[km];
        const float2 Xk = rfft_post(a, b, wk);
        const float2 Xm = rfft_post(b, a, wm);
        x_put<SPEC, M>(lv.fdl, cur, kk, Xk);
        if (km != kk) x_put<SPEC, M>(lv.fdl, cur, km, Xm);
        const float2 Ak = c_mac(tk, Xk, lv_spec_bin<SPEC, M>(lv, slot, 0, kk));
        const float2 Am = c_mac(tm, Xm, lv_spec_bin<SPEC, M>(lv, slot, 0, km));
        z[kk] = irfft_pre(Ak, Am, wk, inv_n);
        if (km != kk) z[km] = irfft_pre(Am, Ak, wm, inv_n);
      }
    }
    __syncthreads();
    fft_inplace<LOG2M, true>(z, tw);
    float* ring = lv.ring + (size_t)slot * lv.R;
    const int rmask = lv.R - 1;
    const long long base = lv.off + j * M;
    for (int m = M / 2 + threadIdx.x; m < M; m += T) {
      const int i = 2 * (m - M / 2);
      ring[(base + i) & rmask] = z[m].x;
      ring[(base + i + 1) & rmask] = z[m].y;
    }
  }
  finish_block(chans, nslots, sync, total, k);
}

template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_commit_kernel(const EngChan* __restrict__ chans, const EngItem* __restrict__ items, int item0, int nitems,
                      const long long* __restrict__ block) {
  const int parity = (int)(*block & 1);  // the coming block
  for (int it = item0 + (int)blockIdx.x; it < item0 + nitems; it += gridDim.x) {
    const EngItem w = items[it];
    if (w.chan < 0 || w.lvl >= 0) continue;
    const EngChan ch = chans[w.chan];
    if (!ch.pending) continue;
    eng_item<LOG2M, SPEC>(ch, w, 1 - ch.active, -1, parity, 1);
  }
}

// Level partial rows of a newly committed IR: the level block j_c = floor(k / p)
// (head still to come at block (j_c + 1) p - 1 >= k) and j_c + 1 (its items
// run from block j_c p on, some perhaps with the old IR), every slice: one
// (item, slice) pair per step of the grid-stride loop, max_slices per item.
template <int LOG2B, int SPEC>
__global__ void __launch_bounds__((1 << LOG2B) / 4)
    eng_level_commit_items_kernel(const EngChan* __restrict__ chans, const EngLevel* __restrict__ levels,
                                  const EngItem* __restrict__ items, int item0, int nitems, int max_slices,
                                  const long long* __restrict__ block) {
  const long long k = *block;
  const long long total = (long long)nitems * max_slices;
  for (long long v = blockIdx.x; v < total; v += gridDim.x) {
    const EngItem w = items[item0 + (int)(v / max_slices)];
    const int slice = (int)(v % max_slices);
    if (w.chan < 0 || w.lvl < 0) continue;
    const EngLevel lv = levels[w.lvl];
    const int pshift = lv.log2N - LOG2B;
    if (slice >= (1 << pshift)) continue;
    const EngChan ch = chans[w.chan];
    if (!ch.pending) continue;
    const long long jc = k >> pshift;
    eng_level_item<LOG2B, SPEC>(lv, w, 1 - ch.active, jc, slice);
    eng_level_item<LOG2B, SPEC>(lv, w, 1 - ch.active, jc + 1, slice);
  }
}

// Output of a newly committed IR for level blocks whose heads have run but
// whose samples reach block k (the coming swap block) or later: block
// j = j_c - 1 - blockIdx.y over every partition, C2R, written into the new IR's
// ring at positions >= k B. Blocks before the stream start write zeros.
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    eng_level_commit_out_kernel(const EngChan* __restrict__ chans, const EngLevel* __restrict__ levels, int log2B,
                                const float2* __restrict__ tw, const long long* __restrict__ block) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  const EngLevel lv = levels[blockIdx.x];
  if (lv.chan < 0) return;
  const EngChan ch = chans[lv.chan];
  if (!ch.pending || !ch.run) return;
  const int slot = 1 - ch.active;
  const long long k = *block, tmin = k << log2B;
  const long long j = (k >> (LOG2M - log2B)) - 1 - (long long)blockIdx.y;
  // first level block with output at or after tmin: off + (j + 1) M > tmin
  const long long d = tmin - lv.off;
  const long long jlo = (d >= 0) ? d / M : -((-d + M - 1) / M);
  if (j < jlo) return;
  float* ring = lv.ring + (size_t)slot * lv.R;
  const int rmask = lv.R - 1;
  const long long base = lv.off + j * M;
  if (j < 0) {
    for (int i = threadIdx.x; i < M; i += T)
      if (base + i >= tmin) ring[(base + i) & rmask] = 0.f;
    return;
  }
  float2* z = sm;
  const int K = lv.K, Kr = lv.Kr;
  const float inv_n = 1.0f / (float)(2 * M);
  for (int kk = threadIdx.x; kk <= M / 2; kk += T) {
    const int km = (kk == 0) ? 0 : M - kk;
    float2 tk = make_float2(0.f, 0.f), tm = tk;
    for (int i = 0; i < K; ++i) {
      const int fs = lv_slot(j - i, Kr);
      const float2 xk = x_bin<SPEC, M>(lv.fdl, fs, kk);
      if (kk == 0) {
        tk = c_mac_dc(tk, xk, lv_spec_bin<SPEC, M>(lv, slot, i, 0));
      } else {
        tk = c_mac(tk, xk, lv_spec_bin<SPEC, M>(lv, slot, i, kk));
        tm = c_mac(tm, x_bin<SPEC, M>(lv.fdl, fs, km), lv_spec_bin<SPEC, M>(lv, slot, i, km));
      }
    }
    if (kk == 0) {
      z[0] = irfft_pre_dc(tk, inv_n);
    } else {
      const float2 wk = __ldg(tw + kk), wm = __ldg(tw + km);
      z[kk] = irfft_pre(tk, tm, wk, inv_n);
      if (km != kk) z[km] = irfft_pre(tm, tk, wm, inv_n);
    }
  }
  __syncthreads();
  fft_inplace<LOG2M, true>(z, tw);
  for (int m = M / 2 + threadIdx.x; m < M; m += T) {
    const int i = 2 * (m - M / 2);
    if (base + i >= tmin) ring[(base + i) & rmask] = z[m].x;
    if (base + i + 1 >= tmin) ring[(base + i + 1) & rmask] = z[m].y;
  }
}

// Marks channel slots [first, first + n) as holding a newly committed IR.
__global__ void eng_mark_pending_kernel(EngChan* __restrict__ chans, int first, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) chans[first + i].pending = 1;
}

// Dynamic shared memory of the block kernel: the head's transform buffers
// (z, z2) and its prefetched tail and H_0 bins (st, sh), M complex values
// each, and with `tw_stage` 3M/2 twiddles. At B / 4 threads per CTA and 1024
// threads per SM that is 128 KB (176 KB) per SM at every block size.
template <int LOG2M>
constexpr int eng_block_smem(bool tw_stage) {
  return (4 * (1 << LOG2M) + (tw_stage ? 3 * (1 << LOG2M) / 2 : 0)) * (int)sizeof(float2);
}

template <int LOG2M, int SPEC>
cudaError_t attrs_t() {
  cudaError_t e = cudaFuncSetAttribute(eng_block_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       eng_block_smem<LOG2M>(true));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(eng_ir_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (1 << LOG2M) * (int)sizeof(float2));
}

template <int LOG2M>
cudaError_t attrs_all() {
  cudaError_t e;
  if ((e = attrs_t<LOG2M, kSpecFP32>()) != cudaSuccess) return e;
  if ((e = attrs_t<LOG2M, kSpecFP16>()) != cudaSuccess) return e;
  if ((e = attrs_t<LOG2M, kSpecBF16>()) != cudaSuccess) return e;
  return attrs_t<LOG2M, kSpecFP24>();
}

// Level kernels of one size: one buffer of M complex values.
template <int LOG2M, int SPEC>
cudaError_t lattrs_t() {
  const int smem = (1 << LOG2M) * (int)sizeof(float2);
  cudaError_t e =
      cudaFuncSetAttribute(eng_level_head_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(eng_level_commit_out_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(eng_level_ir_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <int LOG2M>
cudaError_t lattrs_all() {
  cudaError_t e;
  if ((e = lattrs_t<LOG2M, kSpecFP32>()) != cudaSuccess) return e;
  if ((e = lattrs_t<LOG2M, kSpecFP16>()) != cudaSuccess) return e;
  if ((e = lattrs_t<LOG2M, kSpecBF16>()) != cudaSuccess) return e;
  return lattrs_t<LOG2M, kSpecFP24>();
}

template <int LOG2M, int SPEC>
cudaError_t ir_t(EngChan* chans, const EngUpd* upd, int nupd, int maxP, const float2* tw, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  dim3 grid(maxP, nupd);
  eng_ir_kernel<LOG2M, SPEC><<<grid, S::T, S::M * sizeof(float2), st>>>(chans, upd, tw);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t level_ir_t(EngLevel* levels, const EngLvlUpd* upd, int nupd, int maxK, const float2* tw,
                       cudaStream_t st) {
  using S = FftShape<LOG2M>;
  dim3 grid(maxK, nupd);
  eng_level_ir_kernel<LOG2M, SPEC><<<grid, S::T, S::M * sizeof(float2), st>>>(levels, upd, tw);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t block_t(EngChan* chans, int nslots, const EngItem* items, int nitems, int tail_ctas,
                    const EngLevel* levels, const EngRows& rows, const float2* tw, bool tw_stage, EngSync sync,
                    unsigned total, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_block_kernel<LOG2M, SPEC><<<nslots + tail_ctas, S::T, eng_block_smem<LOG2M>(tw_stage), st>>>(
      chans, nslots, items, nitems, levels, rows, tw, tw_stage ? 1 : 0, sync, total);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t level_head_t(int log2B, EngChan* chans, int nslots, const EngLevel* levels, int nlev,
                         const EngRows& rows, const float2* tw, EngSync sync, unsigned total, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_level_head_kernel<LOG2M, SPEC><<<nlev, S::T, S::M * sizeof(float2), st>>>(chans, nslots, levels, log2B, rows,
                                                                                 tw, sync, total);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t commit_t(const EngChan* chans, const EngItem* items, int item0, int nitems, int grid,
                     const long long* block, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_commit_kernel<LOG2M, SPEC><<<grid, S::T, 0, st>>>(chans, items, item0, nitems, block);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t level_commit_items_t(const EngChan* chans, const EngLevel* levels, const EngItem* items, int item0,
                                 int nitems, int max_slices, int grid, const long long* block, cudaStream_t st) {
  eng_level_commit_items_kernel<LOG2M, SPEC><<<grid, (1 << LOG2M) / 4, 0, st>>>(chans, levels, items, item0, nitems,
                                                                                 max_slices, block);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t level_commit_out_t(int log2B, const EngChan* chans, const EngLevel* levels, int n, int nfl,
                               const float2* tw, const long long* block, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  eng_level_commit_out_kernel<LOG2M, SPEC><<<dim3(n, nfl), S::T, S::M * sizeof(float2), st>>>(chans, levels, log2B,
                                                                                             tw, block);
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

// Level sizes: 2^8 .. 2^kMaxLog2Level (a level block is larger than the
// engine block, which is at least 2^7).
#define ENG_LEVEL_DISPATCH(L2, SP, FN, ...)                               \
  switch ((L2) * 4 + (SP)) {                                              \
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
    case 12 * 4 + 0: return FN<12, 0>(__VA_ARGS__);                       \
    case 12 * 4 + 1: return FN<12, 1>(__VA_ARGS__);                       \
    case 12 * 4 + 2: return FN<12, 2>(__VA_ARGS__);                       \
    case 12 * 4 + 3: return FN<12, 3>(__VA_ARGS__);                       \
    case 13 * 4 + 0: return FN<13, 0>(__VA_ARGS__);                       \
    case 13 * 4 + 1: return FN<13, 1>(__VA_ARGS__);                       \
    case 13 * 4 + 2: return FN<13, 2>(__VA_ARGS__);                       \
    case 13 * 4 + 3: return FN<13, 3>(__VA_ARGS__);                       \
    case 14 * 4 + 0: return FN<14, 0>(__VA_ARGS__);                       \
    case 14 * 4 + 1: return FN<14, 1>(__VA_ARGS__);                       \
    case 14 * 4 + 2: return FN<14, 2>(__VA_ARGS__);                       \
    case 14 * 4 + 3: return FN<14, 3>(__VA_ARGS__);                       \
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
    if ((e = attrs_all<11>()) != cudaSuccess) return e;
    if ((e = lattrs_all<8>()) != cudaSuccess) return e;
    if ((e = lattrs_all<9>()) != cudaSuccess) return e;
    if ((e = lattrs_all<10>()) != cudaSuccess) return e;
    if ((e = lattrs_all<11>()) != cudaSuccess) return e;
    if ((e = lattrs_all<12>()) != cudaSuccess) return e;
    if ((e = lattrs_all<13>()) != cudaSuccess) return e;
    return lattrs_all<14>();
  });
}

cudaError_t eng_launch_ir(int log2B, int spec, EngChan* chans, const EngUpd* upd, int nupd, int maxP,
                          const float2* tw, cudaStream_t st) {
  if (nupd <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, ir_t, chans, upd, nupd, maxP, tw, st);
}

cudaError_t eng_launch_level_ir(int log2N, int spec, EngLevel* levels, const EngLvlUpd* upd, int nupd, int maxK,
                                const float2* tw, cudaStream_t st) {
  if (nupd <= 0) return cudaSuccess;
  ENG_LEVEL_DISPATCH(log2N, spec, level_ir_t, levels, upd, nupd, maxK, tw, st);
}

unsigned eng_block_ctas(int nslots, int tail_ctas) { return (unsigned)(nslots + tail_ctas); }

cudaError_t eng_launch_block(int log2B, int spec, EngChan* chans, int nslots, const EngItem* items, int nitems,
                             int tail_ctas, const EngLevel* levels, const EngRows& rows, const float2* tw,
                             bool tw_stage, EngSync sync, unsigned total, cudaStream_t st) {
  if (nslots <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, block_t, chans, nslots, items, nitems, tail_ctas, levels, rows, tw, tw_stage, sync, total,
               st);
}

cudaError_t eng_launch_level_heads(int log2B, int log2N, int spec, EngChan* chans, int nslots, const EngLevel* levels,
                                   int nlev, const EngRows& rows, const float2* tw, EngSync sync, unsigned total,
                                   cudaStream_t st) {
  if (nlev <= 0) return cudaSuccess;
  ENG_LEVEL_DISPATCH(log2N, spec, level_head_t, log2B, chans, nslots, levels, nlev, rows, tw, sync, total, st);
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

cudaError_t eng_launch_level_commit_items(int log2B, int spec, const EngChan* chans, const EngLevel* levels,
                                          const EngItem* items, int item0, int nitems, int max_slices, int grid,
                                          const long long* block, cudaStream_t st) {
  if (nitems <= 0 || max_slices <= 0) return cudaSuccess;
  ENG_DISPATCH(log2B, spec, level_commit_items_t, chans, levels, items, item0, nitems, max_slices, grid, block, st);
}

cudaError_t eng_launch_level_commit_out(int log2B, int log2N, int spec, const EngChan* chans,
                                        const EngLevel* levels, int first, int n, int nfl, const float2* tw,
                                        const long long* block, cudaStream_t st) {
  if (n <= 0 || nfl <= 0) return cudaSuccess;
  ENG_LEVEL_DISPATCH(log2N, spec, level_commit_out_t, log2B, chans, levels + first, n, nfl, tw, block, st);
}

}  // namespace tanb
