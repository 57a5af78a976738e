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
#include <cstdint>
#include <utility>

#include "tanb_fft.cuh"
#include "tanb_internal.h"

namespace tanb {
namespace {

// Programmatic dependent launch (sm_90+): a kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may begin once every CTA
// of the kernel before it in the stream has executed launch_dependents (or
// exited). The head triggers at once; the tail launched behind it shares no
// data with it, so it never has to wait for the head grid. Without the
// attribute this is a no-op.
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Preferred shared-memory / L1 split (percent of the maximum shared memory)
// of a block's head and tail launches. Both carry the same value: an SM whose
// split has been set for one kernel cannot take CTAs of a kernel that asks
// for another split until it drains, and with the head's dynamic shared
// memory and the tail's small static buffers the driver's own choices differ
// (measured: the tail behind a head with 16 KB of dynamic shared memory ended
// 4 us later than the tail alone; with equal preferences, at the same time).
// 50% holds a head of up to 64 KB beside the tail's CTAs; the 128 KB head of
// 8192-sample blocks takes all of it. A kernel that needs more shared memory
// than its preference gets more regardless.
int pair_carveout(int log2B) { return log2B >= 13 ? 100 : 50; }

// Launch of `kernel`, with programmatic stream serialization when `pdl` is set
// and a preferred shared-memory split when `carveout` >= 0.
template <class... KArgs, class... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                     int carveout, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  int n = 0;
  if (pdl) {
    attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[n].val.programmaticStreamSerializationAllowed = 1;
    ++n;
  }
  if (carveout >= 0) {
    attr[n].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
    attr[n].val.sharedMemCarveout = (unsigned)carveout;
    ++n;
  }
  cfg.attrs = attr;
  cfg.numAttrs = n;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Descriptor sources for the head and tail kernels.
struct DevDesc {
  const ChanCtl* ctl;
  const float* const* in;
  float* const* out;
  __device__ __forceinline__ ChanCtl get_ctl(int c) const { return ctl[c]; }
  __device__ __forceinline__ const float* get_in(int c) const { return in[c]; }
  __device__ __forceinline__ float* get_out(int c) const { return out[c]; }
};
__device__ __forceinline__ ChanCtl unpack_ctl(uint8_t b) {
  return ChanCtl{(b & kCtlRun) ? 1 : 0, (b & kCtlSwap) ? 1 : 0, (b & kCtlSlotCur) ? 1 : 0, (b & kCtlSlotNew) ? 1 : 0};
}
struct ParDesc {
  ParamDesc p;
  __device__ __forceinline__ ChanCtl get_ctl(int c) const { return unpack_ctl(p.c.ctl[c]); }
  __device__ __forceinline__ const float* get_in(int c) const { return p.in[c]; }
  __device__ __forceinline__ float* get_out(int c) const { return p.out[c]; }
};
struct StgDesc {
  StageDesc p;
  __device__ __forceinline__ ChanCtl get_ctl(int c) const { return unpack_ctl(p.c.ctl[c]); }
  __device__ __forceinline__ const float* get_in(int c) const {
    return (p.c.ctl[c] & kCtlHasIn) ? p.in + c * p.stride : nullptr;
  }
  __device__ __forceinline__ float* get_out(int c) const { return p.out + c * p.ostride; }
};
// Channel states only (the tail reads no rows).
struct CtlDesc {
  CtlParam p;
  __device__ __forceinline__ ChanCtl get_ctl(int c) const { return unpack_ctl(p.ctl[c]); }
};


template <int LOG2M>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    ir_spectrum_kernel(DevState s, IrRows ir, const int* __restrict__ chans, const ChanCtl* __restrict__ ctl) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  const int part = blockIdx.x;
  const int row = blockIdx.y;
  const int c = chans[row];
  const int slot = ctl[c].slot_new;
  const float* h = ir.ptrs ? ir.ptrs[row] : ir.base + (size_t)row * ir.stride;
  const long long t0 = (long long)part * M;  // first sample of this partition
  for (int n = threadIdx.x; n < M; n += T) {
    const long long t = t0 + 2 * n;
    float2 v = make_float2(0.f, 0.f);
    if (n < M / 2) {
      if (t < ir.n) v.x = h[t];
      if (t + 1 < ir.n) v.y = h[t + 1];
    }
    sm[n] = v;
  }
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

// 8-point DFT in registers (forward): two 4-point DFTs of the even and odd
// inputs, combined with W_8^q.
__device__ __forceinline__ void dft4_fwd(float2& a, float2& b, float2& c, float2& d) {
  const float2 t0 = c_add(a, c), t1 = c_sub(a, c), t2 = c_add(b, d), t3 = c_sub(b, d);
  const float2 it3 = make_float2(-t3.y, t3.x);
  a = c_add(t0, t2);
  c = c_sub(t0, t2);
  b = c_sub(t1, it3);
  d = c_add(t1, it3);
}
__device__ __forceinline__ void dft8_fwd(float2* v) {
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4_fwd(e0, e1, e2, e3);
  dft4_fwd(o0, o1, o2, o3);
  const float r = 0.70710678118654752f;  // cos(pi/4)
  const float2 w1 = make_float2((o1.x + o1.y) * r, (o1.y - o1.x) * r);     // o1 * W_8
  const float2 w2 = make_float2(o2.y, -o2.x);                               // o2 * W_8^2 = -i
  const float2 w3 = make_float2((o3.y - o3.x) * r, (-o3.y - o3.x) * r);    // o3 * W_8^3
  v[0] = c_add(e0, o0);
  v[4] = c_sub(e0, o0);
  v[1] = c_add(e1, w1);
  v[5] = c_sub(e1, w1);
  v[2] = c_add(e2, w2);
  v[6] = c_sub(e2, w2);
  v[3] = c_add(e3, w3);
  v[7] = c_sub(e3, w3);
}

// IR partition spectra with radix-8 Stockham stages in registers: M / 8
// threads per partition, one shared-memory pass per stage instead of two for
// radix 4 (8192 transforms of 512 points: 32 us against 45 us). When log2 M is
// not a multiple of 3, a radix-2 or radix-4 stage comes first; it reads the
// row directly, where the upper half of the frame is zero. Shared memory is
// padded by one slot per 8 so that the strided stage stores spread over the
// banks. Same inputs, twiddle table and output as ir_spectrum_kernel.
//
// Up to M = 1024 a CTA transforms G partitions side by side (256 threads) and
// first gathers each stage's twiddles into shared memory, ordered so that a
// warp reads consecutive entries: read from the table in global memory, the
// stages' scattered twiddle loads kept the L1 pipe 93% busy (29 us for 8192
// transforms of 512 points, which move 50 MB). The values are the table's, so
// the spectra are the same bit for bit.
template <int LOG2M>
struct IrR8Shape {
  static constexpr int M = 1 << LOG2M, T = M / 8;
  static constexpr int R0 = LOG2M % 3;
  static constexpr int NS0 = R0 == 0 ? 8 : (R0 == 1 ? 2 : 4);  // span after the first stage
  static constexpr bool TWS = T <= 128;                // stage twiddles in shared memory
  static constexpr int G = TWS ? 256 / T : 1;          // partitions per CTA
  static constexpr int THREADS = G * T;
  // the stages' twiddles W^(r k tstep), r = 1..7, k < Ns, stored [stage][r - 1][k]
  // so that a warp's lanes (consecutive k) read consecutive entries
  static constexpr int stage_entries() {
    int n = 0;
    for (int ns = NS0; ns < M; ns *= 8) n += 7 * ns;
    return n;
  }
  static constexpr int TWN = stage_entries();
};

template <int LOG2M>
__global__ void __launch_bounds__(IrR8Shape<LOG2M>::THREADS)
    ir_spectrum_r8_kernel(DevState s, IrRows ir, const int* __restrict__ chans, const ChanCtl* __restrict__ ctl) {
  using Sh = IrR8Shape<LOG2M>;
  constexpr int M = Sh::M, T = Sh::T, G = Sh::G, R0 = Sh::R0;  // first stage radix 2^R0 (1: none)
  constexpr int PADDED = M + M / 8;
  __shared__ float2 sm_all[G * PADDED];
  __shared__ float2 tw_st[Sh::TWS ? Sh::TWN : 1];
  auto pad = [](int i) { return i + (i >> 3); };
  const int grp = (G > 1) ? (int)threadIdx.x / T : 0;
  const int j = (G > 1) ? (int)threadIdx.x % T : (int)threadIdx.x;
  float2* sm = sm_all + grp * PADDED;
  const int part = blockIdx.x * G + grp;
  const bool live = part < s.P;
  const int row = blockIdx.y;
  const int c = chans[row];
  const int slot = ctl[c].slot_new;
  const float* h = ir.ptrs ? ir.ptrs[row] : ir.base + (size_t)row * ir.stride;
  const long long t0 = (long long)part * M;
  const float2* tw = s.tw;
  if constexpr (Sh::TWS) {
    // gathered once per CTA from the table; made visible by the barrier after
    // the first stage
    int base = 0;
    for (int ns = Sh::NS0; ns < M; ns *= 8) {
      const int tstep = (2 * M) / (8 * ns);
      for (int q = threadIdx.x; q < 7 * ns; q += Sh::THREADS) {
        const int r = 1 + q / ns, k = q % ns;
        tw_st[base + q] = __ldg(s.tw + r * k * tstep);
      }
      base += 7 * ns;
    }
  }
  // z[n] = (h[t0 + 2n], h[t0 + 2n + 1]) for n < M / 2, zero above (and for a
  // group past the last partition, which runs the stages for their barriers)
  const bool h8 = (reinterpret_cast<uintptr_t>(h) & 7) == 0;  // t is even: pairs load as one float2
  auto load = [&](int n) {
    float2 v = make_float2(0.f, 0.f);
    if (live && n < M / 2) {
      const long long t = t0 + 2 * n;
      if (h8 && t + 1 < ir.n) {
        v = __ldg(reinterpret_cast<const float2*>(h + t));
      } else {
        if (t < ir.n) v.x = h[t];
        if (t + 1 < ir.n) v.y = h[t + 1];
      }
    }
    return v;
  };
  constexpr int NS0 = Sh::NS0;
  float2 v[8];
  if constexpr (R0 == 0) {
    // radix-8 stage with Ns = 1: inputs j + r M / 8, zero for r >= 4
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = load(j + r * T);
    dft8_fwd(v);
#pragma unroll
    for (int q = 0; q < 8; ++q) sm[pad((j << 3) + q)] = v[q];
  } else if constexpr (R0 == 1) {
    // radix 2, Ns = 1: butterflies b = j + e T (M / 2 of them) pair z[b] with
    // z[b + M / 2] = 0, so both outputs are z[b]
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int b = j + e * T;
      const float2 a = load(b);
      sm[pad(2 * b)] = a;
      sm[pad(2 * b + 1)] = a;
    }
  } else {
    // radix 4, Ns = 1: butterflies b = j + e T (M / 4 of them) on z[b],
    // z[b + M / 4] and two zeros: (a + c, a - i c, a - c, a + i c)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int b = j + e * T;
      const float2 a = load(b), cc = load(b + M / 4);
      sm[pad(4 * b)] = c_add(a, cc);
      sm[pad(4 * b + 1)] = make_float2(a.x + cc.y, a.y - cc.x);
      sm[pad(4 * b + 2)] = c_sub(a, cc);
      sm[pad(4 * b + 3)] = make_float2(a.x - cc.y, a.y + cc.x);
    }
  }
  __syncthreads();
  auto stage = [&](const int Ns, const int tbase) {
    const int k = j & (Ns - 1);
    const int tstep = (2 * M) / (8 * Ns);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const float2 x = sm[pad(j + r * T)];
      if (r == 0) {
        v[r] = x;
      } else if constexpr (Sh::TWS) {
        v[r] = c_mul(x, tw_st[tbase + (r - 1) * Ns + k]);
      } else {
        v[r] = c_mul(x, __ldg(tw + r * k * tstep));
      }
    }
    __syncthreads();
    dft8_fwd(v);
    const int d = ((j - k) << 3) + k;
#pragma unroll
    for (int q = 0; q < 8; ++q) sm[pad(d + q * Ns)] = v[q];
    __syncthreads();
  };
  // Powers of 8 unroll the stages (compile-time spans and twiddle strides);
  // the others keep one loop body, which ptxas fits without spilling.
  if constexpr (R0 == 0) {
    int tb = 0;
#pragma unroll
    for (int Ns = NS0; Ns < M; Ns <<= 3) {
      stage(Ns, tb);
      tb += 7 * Ns;
    }
  } else {
    int tb = 0;
#pragma unroll 1
    for (int Ns = NS0; Ns < M; Ns <<= 3) {
      stage(Ns, tb);
      tb += 7 * Ns;
    }
  }
  if (!live) return;
  float2* H = s.H + h_index(s, c, slot, part);
  for (int k = j; k <= M / 2; k += T) {
    if (k == 0) {
      H[0] = rfft_post_dc(sm[0]);
    } else {
      const int km = M - k;
      const float2 a = sm[pad(k)], b = sm[pad(km)];
      H[k] = rfft_post(a, b, __ldg(s.tw + k));
      if (km != k) H[km] = rfft_post(b, a, __ldg(s.tw + km));
    }
  }
}

// Swap-block output samples i and i + 1 (one packed pair): the new IR's output
// weighted by i / M, the old one's by (M - i) / M (ConvolutionImpl.cpp:1395-1407).
__device__ __forceinline__ float2 crossfade_pair(float2 o, float2 yn, int i, float step, int M) {
  const float a0 = step * (float)i, b0 = step * (float)(M - i);
  const float a1 = step * (float)(i + 1), b1 = step * (float)(M - i - 1);
  return make_float2(yn.x * a0 + o.x * b0, yn.y * a1 + o.y * b1);
}

// Fused PCM epilogue (MixEpi): the channel's output row is in epi.scratch; the
// last head CTA of the channel's group sums the group's rows and converts.
// The counter is an atomic taken once per CTA after a fence: no CTA waits.
template <int M, int T>
__device__ __forceinline__ void mix_epilogue(const MixEpi& epi, int c) {
  __shared__ int last;
  const int g = epi.chan_group[c];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned members = (unsigned)(epi.gstart[g + 1] - epi.gstart[g]);
    last = (atomicAdd(epi.count + g, 1u) == members - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  bool clip = false;
  for (int i = threadIdx.x; i < M; i += T) {
    float sum = 0.f;
    for (int j = epi.gstart[g]; j < epi.gstart[g + 1]; ++j)
      sum = __fadd_rn(sum, __ldcg(epi.scratch + (size_t)epi.gchan[j] * M + i));
    float f = __fmul_rn(sum, epi.out_scale);
    if (f > 32767.f) { f = 32767.f; clip = true; }
    if (f < -32768.f) { f = -32768.f; clip = true; }
    epi.out16[(size_t)g * M + i] = (int16_t)((f != f) ? 0 : __float2int_rz(f));
  }
  if (clip) atomicOr(epi.clip, 1);
  if (threadIdx.x == 0) epi.count[g] = 0u;  // every member has counted itself
}

template <int LOG2M, class D>
__device__ __forceinline__ void head_body(const DevState& s, const D& desc, int cur, int parity, const MixEpi& epi) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T, KP = S::KP;
  extern __shared__ float2 sm[];
  float2* z = sm;       // old / only IR
  float2* z2 = sm + M;  // new IR on a swap block
  const int c = blockIdx.x;
  const ChanCtl cc = desc.get_ctl(c);
  if (!cc.run) return;
  const bool swap = cc.swap != 0;
  const float* x = desc.get_in(c);
  float* y = desc.get_out(c);
  float* prev = s.prev + (size_t)c * M;
  const float2* h0 = s.H + h_index(s, c, cc.slot_cur, 0);
  const float2* h1 = s.H + h_index(s, c, cc.slot_new, 0);
  // tails of this block (partitions >= 2): the IR in use, by block parity, and
  // a pending IR's; partition 1 multiplies X_{k-1}, in the next delay-line slot
  const float2* t0 = s.tail + ((size_t)c * 3 + parity) * M;
  const float2* t1 = s.tail + ((size_t)c * 3 + 2) * M;
  const bool p1 = s.P > 1;
  const float2* xp = s.fdl + ((size_t)c * s.P + (cur + 1) % s.P) * M;

  // Every global load of the prologue is issued before any of them is used,
  // so the block waits for one memory round trip instead of one per phase:
  // first the frame (caller rows may sit in pinned host memory, the longest
  // latency), then the twiddles, then the tail, partitions 0 and 1 and X_{k-1}.
  // frame [x_{k-1}, x_k] packed as complex pairs. 16-byte loads of two pairs
  // when the caller's row allows (history rows and staging rows always do):
  // half the requests, which counts when the row is read over the host bus.
  const bool x_vec = x && (reinterpret_cast<uintptr_t>(x) & 7) == 0;
  const int16_t* x16 = epi.active ? reinterpret_cast<const int16_t*>(x) : nullptr;
  const bool x_v4 = !x16 && (reinterpret_cast<uintptr_t>(x) & 15) == 0;  // also when x is null
  constexpr int E = M / T;
  float2 zr[E];
  if (x_v4) {
    // pair index q = threadIdx.x + j * T holds z[2q], z[2q + 1]
#pragma unroll
    for (int j = 0; j < E / 2; ++j) {
      const int q = threadIdx.x + j * T;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (q < M / 4)
        v = reinterpret_cast<const float4*>(prev)[q];
      else if (x)
        v = reinterpret_cast<const float4*>(x)[q - M / 4];
      zr[2 * j] = make_float2(v.x, v.y);
      zr[2 * j + 1] = make_float2(v.z, v.w);
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int n = threadIdx.x + e * T;
      if (n < M / 2) {
        zr[e] = reinterpret_cast<const float2*>(prev)[n];
      } else if (!x) {
        zr[e] = make_float2(0.f, 0.f);
      } else if (x16) {
        const int k = 2 * (n - M / 2);
        zr[e] = make_float2(__fmul_rn((float)x16[k], epi.in_scale), __fmul_rn((float)x16[k + 1], epi.in_scale));
      } else if (x_vec) {
        zr[e] = reinterpret_cast<const float2*>(x)[n - M / 2];
      } else {
        const float* src = x + 2 * (n - M / 2);
        zr[e] = make_float2(src[0], src[1]);
      }
    }
  }
  // twiddles (staged in shared memory for small transforms), float4 loads
  const float2* tw = s.tw;
  float4 twr[S::TW_SMEM ? E : 1];
  if constexpr (S::TW_SMEM) {
#pragma unroll
    for (int e = 0; e < E; ++e) twr[e] = __ldg(reinterpret_cast<const float4*>(s.tw) + threadIdx.x + e * T);
  }
  // tail and partition 0 of this thread's bin pairs, and the partition-1
  // product's operands; they do not depend on the transform. At 1024 threads
  // (64 registers each) the partition-1 product is taken as its operands
  // arrive, so that the prefetch fits in registers.
  constexpr bool kHoldP1 = T < 1024;
  float2 pt[KP][2], ph[KP][2], px[kHoldP1 ? KP : 1][2], p1h[kHoldP1 ? KP : 1][2];
#pragma unroll
  for (int q = 0; q < KP; ++q) {
    const int k = threadIdx.x + q * T;
    if (k <= M / 2) {
      const int km = (k == 0) ? 0 : M - k;
      pt[q][0] = t0[k];
      pt[q][1] = t0[km];
      ph[q][0] = h0[k];
      ph[q][1] = h0[km];
      if constexpr (kHoldP1) {
        if (p1) {
          px[q][0] = xp[k];
          px[q][1] = xp[km];
          p1h[q][0] = h0[M + k];
          p1h[q][1] = h0[M + km];
        }
      } else if (p1) {
        pt[q][0] = (k == 0) ? c_mac_dc(pt[q][0], xp[0], h0[M]) : c_mac(pt[q][0], xp[k], h0[M + k]);
        if (k != 0) pt[q][1] = c_mac(pt[q][1], xp[km], h0[M + km]);
      }
    }
  }
  if constexpr (S::TW_SMEM) {
    float2* tws = sm + 2 * M;
#pragma unroll
    for (int e = 0; e < E; ++e) reinterpret_cast<float4*>(tws)[threadIdx.x + e * T] = twr[e];
    tw = tws;
  }
  if (x_v4) {
#pragma unroll
    for (int j = 0; j < E / 2; ++j)
      reinterpret_cast<float4*>(z)[threadIdx.x + j * T] =
          make_float4(zr[2 * j].x, zr[2 * j].y, zr[2 * j + 1].x, zr[2 * j + 1].y);
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) z[threadIdx.x + e * T] = zr[e];
  }
  if constexpr (kHoldP1) {
    if (p1) {
#pragma unroll
      for (int q = 0; q < KP; ++q) {
        const int k = threadIdx.x + q * T;
        if (k <= M / 2) {
          pt[q][0] = (k == 0) ? c_mac_dc(pt[q][0], px[q][0], p1h[q][0]) : c_mac(pt[q][0], px[q][0], p1h[q][0]);
          if (k != 0) pt[q][1] = c_mac(pt[q][1], px[q][1], p1h[q][1]);
        }
      }
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < M / 4; q += T)
    reinterpret_cast<float4*>(prev)[q] = reinterpret_cast<const float4*>(z + M / 2)[q];

  fft_inplace<LOG2M, false>(z, tw);

  float2* F = s.fdl + ((size_t)c * s.P + cur) * M;
  const float inv_n = 1.0f / (float)(2 * M);
#pragma unroll
  for (int q = 0; q < KP; ++q) {
    const int k = threadIdx.x + q * T;
    if (k > M / 2) continue;
    if (k == 0) {
      const float2 X = rfft_post_dc(z[0]);
      F[0] = X;
      z[0] = irfft_pre_dc(c_mac_dc(pt[q][0], X, ph[q][0]), inv_n);
      if (swap) {
        const float2 u = p1 ? c_mac_dc(t1[0], xp[0], h1[M]) : t1[0];
        z2[0] = irfft_pre_dc(c_mac_dc(u, X, h1[0]), inv_n);
      }
    } else {
      const int km = M - k;
      const float2 wk = tw[k], wm = tw[km];
      const float2 a = z[k], b = z[km];
      const float2 Xk = rfft_post(a, b, wk);
      const float2 Xm = rfft_post(b, a, wm);
      F[k] = Xk;
      if (km != k) F[km] = Xm;
      const float2 Ak = c_mac(pt[q][0], Xk, ph[q][0]);
      const float2 Am = c_mac(pt[q][1], Xm, ph[q][1]);
      z[k] = irfft_pre(Ak, Am, wk, inv_n);
      if (km != k) z[km] = irfft_pre(Am, Ak, wm, inv_n);
      if (swap) {
        const float2 uk = p1 ? c_mac(t1[k], xp[k], h1[M + k]) : t1[k];
        const float2 um = p1 ? c_mac(t1[km], xp[km], h1[M + km]) : t1[km];
        const float2 Bk = c_mac(uk, Xk, h1[k]);
        const float2 Bm = c_mac(um, Xm, h1[km]);
        z2[k] = irfft_pre(Bk, Bm, wk, inv_n);
        if (km != k) z2[km] = irfft_pre(Bm, Bk, wm, inv_n);
      }
    }
  }
  __syncthreads();
  fft_inplace<LOG2M, true>(z, tw);
  if (swap) fft_inplace<LOG2M, true>(z2, tw);

  // overlap-save: samples [B, 2B) of the circular result are the output
  if (!y) return;
  const float step = 1.0f / (float)M;
  const bool y_vec = (reinterpret_cast<uintptr_t>(y) & 7) == 0;
  if ((reinterpret_cast<uintptr_t>(y) & 15) == 0) {
    // two output pairs (samples 4q .. 4q + 3) per 16-byte store
    for (int q = threadIdx.x; q < M / 4; q += T) {
      const int m = M / 2 + 2 * q;
      float2 o0 = z[m], o1 = z[m + 1];
      if (swap) {
        o0 = crossfade_pair(o0, z2[m], 4 * q, step, M);
        o1 = crossfade_pair(o1, z2[m + 1], 4 * q + 2, step, M);
      }
      reinterpret_cast<float4*>(y)[q] = make_float4(o0.x, o0.y, o1.x, o1.y);
    }
  } else {
    for (int m = M / 2 + threadIdx.x; m < M; m += T) {
      const int i = 2 * (m - M / 2);
      float2 o = z[m];
      if (swap) o = crossfade_pair(o, z2[m], i, step, M);
      if (y_vec) {
        reinterpret_cast<float2*>(y)[i / 2] = o;
      } else {
        y[i] = o.x;
        y[i + 1] = o.y;
      }
    }
  }
  if (epi.active) mix_epilogue<M, T>(epi, c);
}

template <int LOG2M, class D>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    head_kernel(DevState s, const __grid_constant__ D desc, int cur, int parity, MixEpi epi, HeadSignal sig) {
  // The tail launched behind this kernel (the next block's partitions >= 2)
  // shares no data with it and may start at once.
  griddep_launch_dependents();
  head_body<LOG2M>(s, desc, cur, parity, epi);
  if (sig.seq == 0) return;
  // Every CTA, running or not, counts itself once its output stores are
  // visible to the host; the last one raises the flag.
  __threadfence_system();
  __syncthreads();
  if (threadIdx.x == 0 && atomicAdd(sig.count, 1u) == gridDim.x - 1) {
    *sig.count = 0u;
    __threadfence_system();
    *reinterpret_cast<volatile long long*>(sig.flag) = sig.seq;
  }
}

// One float4 = two packed bins. u == 0 holds the packed (DC, Nyquist) pair.
__device__ __forceinline__ float4 mac4(float4 acc, float4 f, float4 h, bool dc) {
  float2 lo = dc ? c_mac_dc(make_float2(acc.x, acc.y), make_float2(f.x, f.y), make_float2(h.x, h.y))
                 : c_mac(make_float2(acc.x, acc.y), make_float2(f.x, f.y), make_float2(h.x, h.y));
  float2 hi = c_mac(make_float2(acc.z, acc.w), make_float2(f.z, f.w), make_float2(h.z, h.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

template <int UX, int SY, int D, class DS>
__global__ void __launch_bounds__(UX* SY)
    tail_kernel(DevState s, const __grid_constant__ DS desc, int which, int cur, int trow) {
  const int c = blockIdx.y;
  const ChanCtl cc = desc.get_ctl(c);
  if (which == 0 ? !cc.run : !cc.swap) return;
  const int slot = (which == 0) ? (cc.swap ? cc.slot_new : cc.slot_cur) : cc.slot_new;
  const int U = s.B >> 1;  // float4 units per partition
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int u = blockIdx.x * UX + tx;
  const int P = s.P;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const bool act = u < U && P > 2;
  const float4* Hc = reinterpret_cast<const float4*>(s.H + h_index(s, c, slot, 0)) + u;
  const float4* Fc = reinterpret_cast<const float4*>(s.fdl + (size_t)c * P * s.B) + u;
  const bool dc = (u == 0);
  if (act) {
    const int nparts = P - 2;  // partitions 2 .. P-1
    const int chunk = (nparts + SY - 1) / SY;
    const int i0 = 2 + ty * chunk;
    const int i1 = min(P, i0 + chunk);
    int i = i0;
    int fs = (cur + i - 1) % P;
    for (; i + D <= i1; i += D) {
      float4 h[D], f[D];
#pragma unroll
      for (int q = 0; q < D; ++q) {
        h[q] = __ldg(Hc + (size_t)(i + q) * U);
        f[q] = __ldg(Fc + (size_t)fs * U);
        fs = (fs + 1 == P) ? 0 : fs + 1;
      }
#pragma unroll
      for (int q = 0; q < D; ++q) acc = mac4(acc, f[q], h[q], dc);
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
  if (u < U) reinterpret_cast<float4*>(s.tail + ((size_t)c * 3 + trow) * s.B)[u] = acc;
}

// ---------------------------------------------------------------------------
// Tail MAC with cp.async.bulk staging. One CTA per (channel, BR-bin slice):
// thread 0 streams, for each chunk of RS partitions, the IR-spectrum and
// delay-line row segments of the slice (BR x 8 bytes each, 16-byte aligned)
// into stage (chunk mod NS) of a shared-memory ring and arms that stage's
// mbarrier with the byte count; all BR/2 threads wait on the barrier, multiply
// and accumulate their two bins from shared memory, then release the stage to
// the next chunk. Up to NS x RS x BR x 16 bytes are in flight per CTA without
// holding them in registers. Waits are bounded: on timeout the kernel records
// kErrBulkWaitTimeout, waits (bounded) for its copies in flight and returns.
// Every copy lands in this CTA's own shared memory and reads this GPU's own memory.

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
  for (int it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int BR, int RS, int NS, class DS>
__global__ void __launch_bounds__(BR / 2)
    tail_bulk_kernel(DevState s, const __grid_constant__ DS desc, int which, int cur, int trow) {
  constexpr int U = BR / 2;                     // threads = float4 units of the slice
  constexpr uint32_t kRowBytes = BR * sizeof(float2);
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  float4* hbuf = reinterpret_cast<float4*>(bulk_smem);             // [NS][RS][U]
  float4* fbuf = hbuf + NS * RS * U;                                // [NS][RS][U]
  uint64_t* bars = reinterpret_cast<uint64_t*>(fbuf + NS * RS * U);  // [NS]
  const int c = blockIdx.y;
  const ChanCtl cc = desc.get_ctl(c);
  if (which == 0 ? !cc.run : !cc.swap) return;
  const int slot = (which == 0) ? (cc.swap ? cc.slot_new : cc.slot_cur) : cc.slot_new;
  const int P = s.P;
  const int bin0 = blockIdx.x * BR;
  const int tid = threadIdx.x;
  const int nparts = P - 2;  // partitions 2 .. P-1
  const int nchunks = (nparts + RS - 1) / RS;
  const float2* Hrow = s.H + h_index(s, c, slot, 0) + bin0;  // + i * B for partition i
  const float2* Frow = s.fdl + (size_t)c * P * s.B + bin0;    // + slot * B

  auto issue = [&](int q) {  // chunk q -> stage q % NS (thread 0 only)
    const int st = q % NS;
    const int i0 = 2 + q * RS;
    const int rows = min(RS, P - i0);
    const uint32_t bar = smem_addr(&bars[st]);
    mbar_expect_tx(bar, 2u * rows * kRowBytes);
    for (int r = 0; r < rows; ++r) {
      const int i = i0 + r;
      const int fs = (cur + i - 1) % P;
      bulk_g2s(smem_addr(hbuf + (st * RS + r) * U), Hrow + (size_t)i * s.B, kRowBytes, bar);
      bulk_g2s(smem_addr(fbuf + (st * RS + r) * U), Frow + (size_t)fs * s.B, kRowBytes, bar);
    }
  };

  if (tid == 0) {
    for (int st = 0; st < NS; ++st) mbar_init(smem_addr(&bars[st]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int q = 0; q < NS && q < nchunks; ++q) issue(q);

  const bool dc = (bin0 == 0 && tid == 0);
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  bool ok = true;
  int q = 0;
  for (; q < nchunks; ++q) {
    const int st = q % NS;
    const uint32_t parity = (uint32_t)(q / NS) & 1u;
    const bool landed = mbar_wait(smem_addr(&bars[st]), parity, s.wait_limit);
    if (__syncthreads_or(!landed)) {  // CTA-uniform decision
      ok = false;
      break;
    }
    const int rows = min(RS, P - (2 + q * RS));
    for (int r = 0; r < rows; ++r)
      acc = mac4(acc, fbuf[(st * RS + r) * U + tid], hbuf[(st * RS + r) * U + tid], dc);
    __syncthreads();  // every thread is done reading stage st
    if (tid == 0 && q + NS < nchunks) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(q + NS);
    }
  }
  if (!ok) {
    // record the failure, then let copies already issued land before exiting
    if (tid == 0) {
      atomicExch(s.err, kErrBulkWaitTimeout);
      for (int r = q; r < nchunks && r < q + NS; ++r)
        mbar_wait(smem_addr(&bars[r % NS]), (uint32_t)(r / NS) & 1u, kBulkWaitLimit);
    }
    __syncthreads();
    return;
  }
  reinterpret_cast<float4*>(s.tail + ((size_t)c * 3 + trow) * s.B + bin0)[tid] = acc;
}

template <int BR, int RS, int NS>
constexpr int bulk_smem_bytes() {
  return 2 * NS * RS * BR * (int)sizeof(float2) + NS * 8;
}

template <int LOG2M>
cudaError_t set_attrs() {
  const int smem = (FftShape<LOG2M>::TW_SMEM ? 4 : 2) * (1 << LOG2M) * (int)sizeof(float2);
  cudaError_t e =
      cudaFuncSetAttribute(head_kernel<LOG2M, DevDesc>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(head_kernel<LOG2M, ParDesc>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(head_kernel<LOG2M, StgDesc>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(ir_spectrum_kernel<LOG2M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (1 << LOG2M) * (int)sizeof(float2));
}

template <int LOG2M>
cudaError_t launch_ir_t(const DevState& s, const IrRows& ir, const int* chans, int nch, const ChanCtl* ctl,
                        cudaStream_t st) {
  using S = FftShape<LOG2M>;
  if constexpr (LOG2M <= 12) {  // the padded buffer of 8192 points exceeds static shared memory
    using R = IrR8Shape<LOG2M>;
    ir_spectrum_r8_kernel<LOG2M><<<dim3((s.P + R::G - 1) / R::G, nch), R::THREADS, 0, st>>>(s, ir, chans, ctl);
  } else {
    ir_spectrum_kernel<LOG2M><<<dim3(s.P, nch), S::T, S::M * sizeof(float2), st>>>(s, ir, chans, ctl);
  }
  return cudaGetLastError();
}

template <int LOG2M>
cudaError_t launch_head_t(const DevState& s, const BlockRef& d, int cur, int parity, cudaStream_t st,
                          const MixEpi& epi, const HeadSignal& sig) {
  using S = FftShape<LOG2M>;
  const size_t smem = (S::TW_SMEM ? 4 : 2) * S::M * sizeof(float2);
  const int cv = pair_carveout(LOG2M);
  if (d.stage)
    return launch_k(head_kernel<LOG2M, StgDesc>, dim3(s.C), dim3(S::T), smem, st, false, cv, s, StgDesc{*d.stage},
                    cur, parity, epi, sig);
  if (d.param)
    return launch_k(head_kernel<LOG2M, ParDesc>, dim3(s.C), dim3(S::T), smem, st, false, cv, s, ParDesc{*d.param},
                    cur, parity, epi, sig);
  return launch_k(head_kernel<LOG2M, DevDesc>, dim3(s.C), dim3(S::T), smem, st, false, cv, s,
                  DevDesc{d.ctl, d.in, d.out}, cur, parity, epi, sig);
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

template <int UX, int SY, int D>
cudaError_t launch_tail_t(const DevState& s, const BlockRef& d, int which, int cur, int trow, cudaStream_t st,
                          bool pdl) {
  const int U = s.B >> 1;
  dim3 grid((U + UX - 1) / UX, s.C);
  dim3 block(UX, SY);
  if (const CtlParam* cp = d.ctl_param())
    return launch_k(tail_kernel<UX, SY, D, CtlDesc>, grid, block, 0, st, pdl, pair_carveout(s.log2B), s,
                    CtlDesc{*cp}, which, cur, trow);
  return launch_k(tail_kernel<UX, SY, D, DevDesc>, grid, block, 0, st, pdl, pair_carveout(s.log2B), s,
                  DevDesc{d.ctl, d.in, d.out}, which,
                  cur, trow);
}

template <int BR, int RS, int NS>
cudaError_t launch_bulk_t(const DevState& s, const BlockRef& d, int which, int cur, int trow, cudaStream_t st,
                          bool pdl) {
  if (s.B % BR != 0) return cudaErrorInvalidValue;
  constexpr int smem = bulk_smem_bytes<BR, RS, NS>();
  static OncePerDevice once;
  const cudaError_t attr = once.run([] {
    cudaError_t e = cudaFuncSetAttribute(tail_bulk_kernel<BR, RS, NS, DevDesc>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(tail_bulk_kernel<BR, RS, NS, CtlDesc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem);
  });
  if (attr != cudaSuccess) return attr;
  dim3 grid(s.B / BR, s.C);
  if (const CtlParam* cp = d.ctl_param())
    return launch_k(tail_bulk_kernel<BR, RS, NS, CtlDesc>, grid, dim3(BR / 2), smem, st, pdl, pair_carveout(s.log2B), s, CtlDesc{*cp},
                    which, cur, trow);
  return launch_k(tail_bulk_kernel<BR, RS, NS, DevDesc>, grid, dim3(BR / 2), smem, st, pdl, pair_carveout(s.log2B), s,
                  DevDesc{d.ctl, d.in, d.out}, which, cur, trow);
}

using TailLauncher = cudaError_t (*)(const DevState&, const BlockRef&, int, int, int, cudaStream_t, bool);
struct TailEntry {
  MacTiling t;
  TailLauncher fn;
};
// The tilings the autotuner chooses among.
const TailEntry kTail[] = {
    {{32, 8, 4}, launch_tail_t<32, 8, 4>},   {{16, 16, 4}, launch_tail_t<16, 16, 4>},
    {{32, 8, 8}, launch_tail_t<32, 8, 8>},   {{32, 16, 4}, launch_tail_t<32, 16, 4>},
    {{32, 16, 8}, launch_tail_t<32, 16, 8>}, {{64, 4, 4}, launch_tail_t<64, 4, 4>},
    {{64, 8, 4}, launch_tail_t<64, 8, 4>},   {{64, 8, 8}, launch_tail_t<64, 8, 8>},
    {{128, 2, 8}, launch_tail_t<128, 2, 8>}, {{32, 32, 4}, launch_tail_t<32, 32, 4>},
    {{16, 32, 8}, launch_tail_t<16, 32, 8>}, {{64, 16, 2}, launch_tail_t<64, 16, 2>},
    // cp.async.bulk pipelines: {BR/2, stages, rows per stage, kind 1}
    {{32, 4, 8, 1}, launch_bulk_t<64, 8, 4>},   {{64, 4, 8, 1}, launch_bulk_t<128, 8, 4>},
    {{64, 6, 4, 1}, launch_bulk_t<128, 4, 6>},  {{128, 4, 4, 1}, launch_bulk_t<256, 4, 4>},
    {{64, 8, 8, 1}, launch_bulk_t<128, 8, 8>},  {{128, 3, 8, 1}, launch_bulk_t<256, 8, 3>},
};
constexpr int kTailCount = sizeof(kTail) / sizeof(kTail[0]);

}  // namespace

cudaError_t prepare_kernels() {
  static OncePerDevice once;
  return once.run([] {
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
  });
}

cudaError_t launch_ir_spectrum(const DevState& s, const IrRows& ir, const int* chans, int nch,
                               const ChanCtl* ctl, cudaStream_t st) {
  if (nch <= 0) return cudaSuccess;
  TANB_DISPATCH_LOG2(s.log2B, launch_ir_t, s, ir, chans, nch, ctl, st);
}

cudaError_t launch_head(const DevState& s, const BlockRef& d, int cur, int parity, cudaStream_t st,
                        const MixEpi& epi, const HeadSignal& sig) {
  TANB_DISPATCH_LOG2(s.log2B, launch_head_t, s, d, cur, parity, st, epi, sig);
}

cudaError_t launch_tail(const DevState& s, const BlockRef& d, int which, int cur, int trow, MacTiling t,
                        cudaStream_t st, bool pdl) {
  if (s.P <= 2) return cudaSuccess;
  for (int i = 0; i < kTailCount; ++i)
    if (kTail[i].t.ux == t.ux && kTail[i].t.sy == t.sy && kTail[i].t.depth == t.depth &&
        kTail[i].t.kind == t.kind)
      return kTail[i].fn(s, d, which, cur, trow, st, pdl);
  return cudaErrorInvalidValue;
}

int mac_tiling_count() { return kTailCount; }

MacTiling mac_tiling(int index) { return kTail[index].t; }

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
