// Non-uniformly partitioned convolution (the TAN_CONVOLUTION_METHOD_*_NONUNIFORM
// family; the reference's CPU variant is ConvolutionImpl.cpp:224-246 and
// 2416-2428, its GPU two-stream engine tan/tanlibrary/src/Graal2/Reverberate.cpp).
//
// The IR is cut into levels l = 0..NL-1: level l has block N_l (a power of two,
// N_0 = the base block B0) and K_l partitions covering IR taps
// [o_l, o_l + K_l N_l), o_0 = 0, o_l = sum_{m<l} K_m N_m, with o_l >= N_l for
// l >= 1. Each level is a uniformly partitioned overlap-save convolution of the
// input with its IR segment, computed once per N_l samples, when its input
// block completes; its N_l outputs land at absolute samples
// [o_l + j N_l, o_l + (j+1) N_l), never before the base block that follows,
// so only level 0 is on a block's critical path. Per base block k:
//   1. the input block goes into a per-channel input ring;
//   2. level 0: R2C of its 2B0 frame, multiply with partitions 0 and 1 (the
//      new spectrum and the previous one), add its precomputed tail, C2R, add
//      the output ring's block k (contributions of the larger levels,
//      computed in earlier blocks) -> output; clear them;
//   3. level 0's tail (partitions 2..K-1) for block k+1, when K > 2;
//   4. every level whose block completes: head (as 2, adding into the output
//      ring at its delayed position) and tail (as 3).
// The kernels of a block are launched in level order, for the levels that are
// due at that block only: with power-of-two block sizes the set of due levels
// follows from the block index, so each set is one CUDA graph captured at
// creation and the host launches the one for the block (the kernels check the
// same condition and exit when their level is not due). Contributions to a
// ring sample are added in a fixed order,
// so results are deterministic. IR spectra are FP32, FP16 or BF16 with
// per-partition power-of-two scales; accumulation is FP32.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdarg>
#include <map>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/tanb.h"
#include "tanb_fft.cuh"
#include "tanb_internal.h"

namespace tanb {
namespace {

constexpr int kMaxLevels = 16;

struct NuLevel {
  int log2N;
  int K;            // partitions
  long long off;    // IR offset o_l
  void* H;          // [C][K][N] spectra
  float* scale;     // [C][K] (FP16 / BF16)
  float2* fdl;      // [C][K][N]
  float2* tail;     // [C][N]
};

struct NuDev {
  int C;
  int B0;
  int spec;
  int nl;
  int rin;          // input ring length (power of two)
  int rout;         // output ring length (power of two)
  float* in_ring;   // [C][rin]
  float* out_ring;  // [C][rout]
  long long* k;     // base block counter (device)
  const float2* tw[kMaxLevels];  // twiddles per level (2 N_l entries)
  NuLevel lv[kMaxLevels];
};

template <int SPEC>
__device__ __forceinline__ float2 spec_get(const void* p, size_t k) {
  if constexpr (SPEC == 0) return reinterpret_cast<const float2*>(p)[k];
  else if constexpr (SPEC == 1) return __half22float2(reinterpret_cast<const __half2*>(p)[k]);
  else return __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(p)[k]);
}

template <int SPEC>
__device__ __forceinline__ void spec_put(void* p, size_t k, float2 v) {
  if constexpr (SPEC == 0) reinterpret_cast<float2*>(p)[k] = v;
  else if constexpr (SPEC == 1) reinterpret_cast<__half2*>(p)[k] = __float22half2_rn(v);
  else reinterpret_cast<__nv_bfloat162*>(p)[k] = __float22bfloat162_rn(v);
}

// Level block j completes at base block k when (k+1) B0 is a multiple of N.
__device__ __forceinline__ bool level_due(long long k, int B0, int N, long long* j) {
  const long long end = (k + 1) * (long long)B0;
  if (end % N) return false;
  *j = end / N - 1;
  return true;
}

// Delay-line slot of the level block j's spectrum: K-1 - (j mod K).
__device__ __forceinline__ int slot_of(long long j, int K) { return (int)(K - 1 - (j % K)); }

__global__ void nu_input_kernel(NuDev d, const float* __restrict__ in, int ld) {
  const int c = blockIdx.y;
  const long long k = *d.k;
  const float* x = in ? in + (size_t)c * ld : nullptr;
  float* ring = d.in_ring + (size_t)c * d.rin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.B0; i += gridDim.x * blockDim.x)
    ring[(k * d.B0 + i) & (d.rin - 1)] = x ? x[i] : 0.f;
}

// Head of level L (template LOG2M = log2 N_L). L == 0 writes the block's
// output (adding and clearing the output ring's block); L >= 1 adds into the
// output ring at its delayed position.
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    nu_head_kernel(NuDev d, int L, float* __restrict__ out, int ld) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  const int c = blockIdx.x;
  const long long k = *d.k;
  long long j;
  if (!level_due(k, d.B0, M, &j)) return;
  const NuLevel lv = d.lv[L];
  const float2* tw = d.tw[L];
  float2* z = sm;
  // frame: input samples [(j-1) M, (j+1) M) from the ring
  const float* ring = d.in_ring + (size_t)c * d.rin;
  const long long s0 = (j - 1) * (long long)M;
  for (int n = threadIdx.x; n < M; n += T) {
    const long long a = s0 + 2 * n;
    z[n] = (a < 0) ? make_float2(0.f, 0.f)
                   : make_float2(ring[a & (d.rin - 1)], ring[(a + 1) & (d.rin - 1)]);
  }
  __syncthreads();
  fft_inplace<LOG2M, false>(z, tw);
  const int K = lv.K;
  const int cur = slot_of(j, K);
  float2* F = lv.fdl + ((size_t)c * K + cur) * M;
  const size_t h0 = (size_t)c * K * M;
  const float s0c = (SPEC != 0) ? lv.scale[(size_t)c * K] : 1.f;
  const float2* t0 = lv.tail + (size_t)c * M;
  // partition 1 (X_{j-1} * H_1) is taken here; the tail holds partitions >= 2
  const bool p1 = K > 1 && j > 0;
  const float2* Fp = lv.fdl + ((size_t)c * K + (p1 ? slot_of(j - 1, K) : 0)) * M;
  const float s1c = (SPEC != 0 && K > 1) ? lv.scale[(size_t)c * K + 1] : 1.f;
  const float inv_n = 1.0f / (float)(2 * M);
  for (int kk = threadIdx.x; kk <= M / 2; kk += T) {
    if (kk == 0) {
      const float2 X = rfft_post_dc(z[0]);
      float2 t = t0[0];
      if (p1) {
        float2 h1 = spec_get<SPEC>(lv.H, h0 + M);
        h1.x *= s1c;
        h1.y *= s1c;
        t = c_mac_dc(t, Fp[0], h1);
      }
      F[0] = X;
      float2 h = spec_get<SPEC>(lv.H, h0);
      h.x *= s0c;
      h.y *= s0c;
      z[0] = irfft_pre_dc(c_mac_dc(t, X, h), inv_n);
    } else {
      const int km = M - kk;
      const float2 wk = tw[kk], wm = tw[km];
      const float2 a = z[kk], b = z[km];
      const float2 Xk = rfft_post(a, b, wk);
      const float2 Xm = rfft_post(b, a, wm);
      float2 tk = t0[kk], tm = t0[km];
      if (p1) {
        float2 gk = spec_get<SPEC>(lv.H, h0 + M + kk), gm = spec_get<SPEC>(lv.H, h0 + M + km);
        gk.x *= s1c; gk.y *= s1c; gm.x *= s1c; gm.y *= s1c;
        tk = c_mac(tk, Fp[kk], gk);
        tm = c_mac(tm, Fp[km], gm);
      }
      F[kk] = Xk;
      if (km != kk) F[km] = Xm;
      float2 hk = spec_get<SPEC>(lv.H, h0 + kk), hm = spec_get<SPEC>(lv.H, h0 + km);
      hk.x *= s0c; hk.y *= s0c; hm.x *= s0c; hm.y *= s0c;
      const float2 Ak = c_mac(tk, Xk, hk);
      const float2 Am = c_mac(tm, Xm, hm);
      z[kk] = irfft_pre(Ak, Am, wk, inv_n);
      if (km != kk) z[km] = irfft_pre(Am, Ak, wm, inv_n);
    }
  }
  __syncthreads();
  fft_inplace<LOG2M, true>(z, tw);
  float* oring = d.out_ring + (size_t)c * d.rout;
  if (L == 0) {
    // base block k: this level's samples plus the ring's, then clear the ring
    float* y = out + (size_t)c * ld;
    const long long t0s = k * (long long)d.B0;
    for (int m = M / 2 + threadIdx.x; m < M; m += T) {
      const int i = 2 * (m - M / 2);
      const long long p0 = (t0s + i) & (d.rout - 1), p1 = (t0s + i + 1) & (d.rout - 1);
      y[i] = z[m].x + oring[p0];
      y[i + 1] = z[m].y + oring[p1];
      oring[p0] = 0.f;
      oring[p1] = 0.f;
    }
  } else {
    const long long base = lv.off + j * (long long)M;
    for (int m = M / 2 + threadIdx.x; m < M; m += T) {
      const int i = 2 * (m - M / 2);
      oring[(base + i) & (d.rout - 1)] += z[m].x;
      oring[(base + i + 1) & (d.rout - 1)] += z[m].y;
    }
  }
}

// Tail of level L for its next block: sum_{i=2}^{K-1} FDL[(cur + i - 1) mod K] * H_i
// (cur = slot of the block just inserted); partition 1 belongs to the head,
// so the tail reads no spectrum the head writes. One CTA per (channel, 2*UX-bin
// slice), partitions split over SY warps, reduced in shared memory.
template <int SPEC, int UX, int SY>
__global__ void __launch_bounds__(UX* SY) nu_tail_kernel(NuDev d, int L, int log2N) {
  const int N = 1 << log2N;
  const long long k = *d.k;
  long long j;
  if (!level_due(k, d.B0, N, &j)) return;
  const NuLevel lv = d.lv[L];
  const int c = blockIdx.y;
  const int U = N >> 1;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int u = blockIdx.x * UX + tx;
  const int K = lv.K;
  float2 a0 = make_float2(0.f, 0.f), a1 = a0;
  if (u < U && K > 2) {
    const int cur = slot_of(j, K);
    const int nparts = K - 2;
    const int chunk = (nparts + SY - 1) / SY;
    const int i0 = 2 + ty * chunk, i1 = min(K, i0 + chunk);
    const float4* Fc = reinterpret_cast<const float4*>(lv.fdl + (size_t)c * K * N) + u;
    const bool dc = (u == 0);
    int fs = (cur + i0 - 1) % K;
    for (int i = i0; i < i1; ++i) {
      const float4 f = __ldg(Fc + (size_t)fs * U);
      fs = (fs + 1 == K) ? 0 : fs + 1;
      const size_t hb = ((size_t)c * K + i) * N + 2 * (size_t)u;
      float2 ha = spec_get<SPEC>(lv.H, hb), hb2 = spec_get<SPEC>(lv.H, hb + 1);
      if (SPEC != 0) {
        const float s = __ldg(lv.scale + (size_t)c * K + i);
        ha.x *= s; ha.y *= s; hb2.x *= s; hb2.y *= s;
      }
      const float2 fa = make_float2(f.x, f.y), fb = make_float2(f.z, f.w);
      a0 = dc ? c_mac_dc(a0, fa, ha) : c_mac(a0, fa, ha);
      a1 = c_mac(a1, fb, hb2);
    }
  }
  __shared__ float4 red[SY][UX];
  red[ty][tx] = make_float4(a0.x, a0.y, a1.x, a1.y);
  __syncthreads();
  if (ty != 0 || u >= U) return;
  float4 acc = red[0][tx];
  for (int q = 1; q < SY; ++q) {
    const float4 r = red[q][tx];
    acc.x += r.x; acc.y += r.y; acc.z += r.z; acc.w += r.w;
  }
  reinterpret_cast<float4*>(lv.tail + (size_t)c * N)[u] = acc;
}

__global__ void nu_step_kernel(NuDev d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *d.k += 1;
}

// IR spectra of level L: one CTA per (partition, channel); ir rows [C][stride].
template <int LOG2M, int SPEC>
__global__ void __launch_bounds__(FftShape<LOG2M>::T)
    nu_ir_kernel(NuDev d, int L, const float* __restrict__ ir, long long stride, long long n) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T;
  extern __shared__ float2 sm[];
  __shared__ float red[32];
  const NuLevel lv = d.lv[L];
  const float2* tw = d.tw[L];
  const int part = blockIdx.x, c = blockIdx.y;
  const long long t0 = lv.off + (long long)part * M;
  const float* h = ir + (size_t)c * stride;
  for (int q = threadIdx.x; q < M; q += T) {
    const long long a = t0 + 2 * q;
    sm[q] = (q < M / 2) ? make_float2(a < n ? h[a] : 0.f, a + 1 < n ? h[a + 1] : 0.f) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_inplace<LOG2M, false>(sm, tw);
  for (int kk = threadIdx.x; kk <= M / 2; kk += T) {
    if (kk == 0) {
      sm[0] = rfft_post_dc(sm[0]);
    } else {
      const int km = M - kk;
      const float2 a = sm[kk], b = sm[km];
      const float2 Xk = rfft_post(a, b, tw[kk]);
      const float2 Xm = rfft_post(b, a, tw[km]);
      sm[kk] = Xk;
      if (km != kk) sm[km] = Xm;
    }
  }
  __syncthreads();
  float scale = 1.f;
  if constexpr (SPEC != 0) {
    float mx = 0.f;
    for (int q = threadIdx.x; q < M; q += T) mx = fmaxf(mx, fmaxf(fabsf(sm[q].x), fabsf(sm[q].y)));
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
    int e = 0;
    if (mx > 0.f) {
      frexpf(mx, &e);
      e -= 15;
    }
    // a partition of denormal samples: keep the scale a normal number (2^-149
    // would round to zero and its inverse overflow)
    e = e < -126 ? -126 : e;
    scale = ldexpf(1.f, e);
    if (threadIdx.x == 0) lv.scale[(size_t)c * lv.K + part] = scale;
  }
  const float inv = 1.f / scale;
  for (int q = threadIdx.x; q < M; q += T)
    spec_put<SPEC>(lv.H, ((size_t)c * lv.K + part) * M + q, make_float2(sm[q].x * inv, sm[q].y * inv));
}

// --- launchers ---------------------------------------------------------------
template <int LOG2M, int SPEC>
cudaError_t head_t(const NuDev& d, int L, float* out, int ld, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  static OncePerDevice once;
  const cudaError_t attr = once.run([] {
    return cudaFuncSetAttribute(nu_head_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                S::M * (int)sizeof(float2));
  });
  if (attr != cudaSuccess) return attr;
  nu_head_kernel<LOG2M, SPEC><<<d.C, S::T, S::M * sizeof(float2), st>>>(d, L, out, ld);
  return cudaGetLastError();
}

template <int LOG2M, int SPEC>
cudaError_t ir_t(const NuDev& d, int L, const float* ir, long long stride, long long n, cudaStream_t st) {
  using S = FftShape<LOG2M>;
  static OncePerDevice once;
  const cudaError_t attr = once.run([] {
    return cudaFuncSetAttribute(nu_ir_kernel<LOG2M, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                S::M * (int)sizeof(float2));
  });
  if (attr != cudaSuccess) return attr;
  dim3 grid(d.lv[L].K, d.C);
  nu_ir_kernel<LOG2M, SPEC><<<grid, S::T, S::M * sizeof(float2), st>>>(d, L, ir, stride, n);
  return cudaGetLastError();
}

#define NU_DISPATCH(L2, SP, FN, ...)                  \
  switch ((L2) * 4 + (SP)) {                          \
    case 5 * 4 + 0: return FN<5, 0>(__VA_ARGS__);     \
    case 5 * 4 + 1: return FN<5, 1>(__VA_ARGS__);     \
    case 5 * 4 + 2: return FN<5, 2>(__VA_ARGS__);     \
    case 6 * 4 + 0: return FN<6, 0>(__VA_ARGS__);     \
    case 6 * 4 + 1: return FN<6, 1>(__VA_ARGS__);     \
    case 6 * 4 + 2: return FN<6, 2>(__VA_ARGS__);     \
    case 7 * 4 + 0: return FN<7, 0>(__VA_ARGS__);     \
    case 7 * 4 + 1: return FN<7, 1>(__VA_ARGS__);     \
    case 7 * 4 + 2: return FN<7, 2>(__VA_ARGS__);     \
    case 8 * 4 + 0: return FN<8, 0>(__VA_ARGS__);     \
    case 8 * 4 + 1: return FN<8, 1>(__VA_ARGS__);     \
    case 8 * 4 + 2: return FN<8, 2>(__VA_ARGS__);     \
    case 9 * 4 + 0: return FN<9, 0>(__VA_ARGS__);     \
    case 9 * 4 + 1: return FN<9, 1>(__VA_ARGS__);     \
    case 9 * 4 + 2: return FN<9, 2>(__VA_ARGS__);     \
    case 10 * 4 + 0: return FN<10, 0>(__VA_ARGS__);   \
    case 10 * 4 + 1: return FN<10, 1>(__VA_ARGS__);   \
    case 10 * 4 + 2: return FN<10, 2>(__VA_ARGS__);   \
    case 11 * 4 + 0: return FN<11, 0>(__VA_ARGS__);   \
    case 11 * 4 + 1: return FN<11, 1>(__VA_ARGS__);   \
    case 11 * 4 + 2: return FN<11, 2>(__VA_ARGS__);   \
    case 12 * 4 + 0: return FN<12, 0>(__VA_ARGS__);   \
    case 12 * 4 + 1: return FN<12, 1>(__VA_ARGS__);   \
    case 12 * 4 + 2: return FN<12, 2>(__VA_ARGS__);   \
    case 13 * 4 + 0: return FN<13, 0>(__VA_ARGS__);   \
    case 13 * 4 + 1: return FN<13, 1>(__VA_ARGS__);   \
    case 13 * 4 + 2: return FN<13, 2>(__VA_ARGS__);   \
    default: return cudaErrorInvalidValue;            \
  }

cudaError_t launch_nu_head(const NuDev& d, int L, float* out, int ld, cudaStream_t st) {
  NU_DISPATCH(d.lv[L].log2N, d.spec, head_t, d, L, out, ld, st);
}

cudaError_t launch_nu_ir(const NuDev& d, int L, const float* ir, long long stride, long long n, cudaStream_t st) {
  NU_DISPATCH(d.lv[L].log2N, d.spec, ir_t, d, L, ir, stride, n, st);
}

template <int SPEC>
cudaError_t tail_s(const NuDev& d, int L, cudaStream_t st) {
  const int N = 1 << d.lv[L].log2N, U = N / 2;
  if (d.lv[L].K <= 1) return cudaSuccess;
  if (U >= 64) {
    dim3 grid(U / 64, d.C), block(64, 8);
    nu_tail_kernel<SPEC, 64, 8><<<grid, block, 0, st>>>(d, L, d.lv[L].log2N);
  } else {
    dim3 grid(1, d.C), block(32, 16);  // N <= 64: one CTA row covers every bin pair
    nu_tail_kernel<SPEC, 32, 16><<<grid, block, 0, st>>>(d, L, d.lv[L].log2N);
  }
  return cudaGetLastError();
}

cudaError_t launch_nu_tail(const NuDev& d, int L, cudaStream_t st) {
  // two partitions or fewer: no tail (the head takes partitions 0 and 1); the
  // level's tail row keeps the zeros it was allocated with
  if (d.lv[L].K <= 2) return cudaSuccess;
  switch (d.spec) {
    case 0: return tail_s<0>(d, L, st);
    case 1: return tail_s<1>(d, L, st);
    default: return tail_s<2>(d, L, st);
  }
}

int32_t nfail(int32_t code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}

#define NU_CUDA(expr)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return nfail(e_ == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL,   \
                   "%s failed: %s", #expr, cudaGetErrorString(e_));                   \
  } while (0)

size_t pow2_at_least(size_t x) {
  size_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace
}  // namespace tanb

struct tanb_nu {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  tanb::NuDev d{};
  int L = 0;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  float* d_in = nullptr;    // [C][B0] staging
  float* d_out = nullptr;   // [C][B0]
  float* h_in = nullptr;    // pinned
  float* h_out = nullptr;
  float* d_ir = nullptr;    // [C][L] staging for set_response
  long long k = 0;          // host mirror of the base block counter
  size_t dev_bytes = 0;
  // host-buffer block graphs, one per set of due levels (bit l: level l)
  std::map<unsigned, cudaGraphExec_t> graphs;
  cudaEvent_t ev_out = nullptr;
};

namespace {

using tanb::nfail;

cudaError_t nu_alloc(tanb_nu* v, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return e;
  v->allocs.push_back(*p);
  v->dev_bytes += bytes;
  return cudaMemsetAsync(*p, 0, bytes, v->stream);
}

void nu_free(tanb_nu* v) {
  if (v->stream) cudaStreamSynchronize(v->stream);
  for (auto& kv : v->graphs) cudaGraphExecDestroy(kv.second);
  v->graphs.clear();
  for (void* p : v->allocs) cudaFree(p);
  v->allocs.clear();
  cudaFreeHost(v->h_in);
  cudaFreeHost(v->h_out);
  if (v->ev_out) cudaEventDestroy(v->ev_out);
  if (v->stream) cudaStreamDestroy(v->stream);
}

// Levels whose block completes with base block k (bit l: level l; level 0,
// whose block is the base block, always): N_l divides (k + 1) B0. With
// power-of-two block sizes the pattern repeats every max N_l / B0 blocks.
unsigned due_mask(const tanb::NuDev& d, long long k) {
  unsigned m = 0;
  for (int l = 0; l < d.nl; ++l)
    if (((k + 1) * (long long)d.B0) % (1LL << d.lv[l].log2N) == 0) m |= 1u << l;
  return m;
}

// Kernels of one base block in level order, for the levels in `due` (the
// kernels check the same condition on the device counter); input from `in`
// ([C][ld] or null).
cudaError_t enqueue_nu_block(tanb_nu* v, const float* in, float* out, int ld, bool host, unsigned due) {
  const tanb::NuDev& d = v->d;
  cudaError_t r;
  if (host && (r = cudaMemcpyAsync(v->d_in, v->h_in, (size_t)d.C * d.B0 * sizeof(float), cudaMemcpyHostToDevice,
                                   v->stream)) != cudaSuccess)
    return r;
  dim3 gi((d.B0 + 255) / 256, d.C);
  tanb::nu_input_kernel<<<gi, 256, 0, v->stream>>>(d, in, ld);
  if ((r = cudaGetLastError()) != cudaSuccess) return r;
  if ((r = tanb::launch_nu_head(d, 0, out, ld, v->stream)) != cudaSuccess) return r;
  if (host) {
    if ((r = cudaMemcpyAsync(v->h_out, v->d_out, (size_t)d.C * d.B0 * sizeof(float), cudaMemcpyDeviceToHost,
                             v->stream)) != cudaSuccess)
      return r;
    if ((r = cudaEventRecordWithFlags(v->ev_out, v->stream, cudaEventRecordExternal)) != cudaSuccess) return r;
  }
  if ((r = tanb::launch_nu_tail(d, 0, v->stream)) != cudaSuccess) return r;
  for (int l = 1; l < d.nl; ++l) {
    if (!(due >> l & 1u)) continue;
    if ((r = tanb::launch_nu_head(d, l, nullptr, 0, v->stream)) != cudaSuccess) return r;
    if ((r = tanb::launch_nu_tail(d, l, v->stream)) != cudaSuccess) return r;
  }
  tanb::nu_step_kernel<<<1, 32, 0, v->stream>>>(d);
  return cudaGetLastError();
}

// The host-buffer block as a CUDA graph holding only the due levels' kernels,
// one graph per set of due levels, captured once. Creation calls this for
// every set that one period of the schedule produces, so that module loading,
// instantiation and the upload of the graphs to the device are not paid by
// audio blocks.
cudaError_t ensure_graph(tanb_nu* v, unsigned due) {
  if (v->graphs.count(due)) return cudaSuccess;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  cudaError_t r = cudaStreamBeginCapture(v->stream, cudaStreamCaptureModeThreadLocal);
  if (r != cudaSuccess) return r;
  r = enqueue_nu_block(v, v->d_in, v->d_out, v->d.B0, true, due);
  cudaError_t r2 = cudaStreamEndCapture(v->stream, &g);
  if (r == cudaSuccess) r = r2;
  if (r == cudaSuccess) r = cudaGraphInstantiate(&ge, g, 0);
  if (g) cudaGraphDestroy(g);
  if (r == cudaSuccess) r = cudaGraphUpload(ge, v->stream);
  if (r == cudaSuccess)
    v->graphs[due] = ge;
  else if (ge)
    cudaGraphExecDestroy(ge);
  return r;
}

cudaError_t ensure_graphs(tanb_nu* v) {
  long long period = 1;
  for (int l = 0; l < v->d.nl; ++l) period = std::max(period, (1LL << v->d.lv[l].log2N) / v->d.B0);
  for (long long k = 0; k < period; ++k) {
    const cudaError_t r = ensure_graph(v, due_mask(v->d, k));
    if (r != cudaSuccess) return r;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

int32_t tanb_nu_schedule(uint32_t ir_length, uint32_t base_block, uint32_t max_block, uint32_t* nlevels,
                         uint32_t* level_block, uint32_t* level_parts) {
  if (!nlevels || !level_block || !level_parts) return nfail(TANB_INVALID_POINTER, "null argument");
  if (base_block < 32 || (base_block & (base_block - 1)) || max_block < base_block ||
      (max_block & (max_block - 1)) || max_block > 16384 || ir_length == 0)
    return nfail(TANB_INVALID_ARG, "blocks must be powers of two, 32 <= base <= max <= 16384");
  // two partitions per size while doubling, the largest size takes the rest
  uint32_t n = 0;
  long long off = 0;
  for (uint32_t N = base_block; N < max_block && off < (long long)ir_length; N <<= 1) {
    if (n + 1 >= (uint32_t)tanb::kMaxLevels) break;
    level_block[n] = N;
    level_parts[n] = 2;
    off += 2LL * N;
    ++n;
  }
  if (off < (long long)ir_length) {
    const uint32_t N = (n == 0) ? base_block : std::min<uint32_t>(max_block, level_block[n - 1] * 2);
    level_block[n] = N;
    level_parts[n] = (uint32_t)((ir_length - off + N - 1) / N);
    ++n;
  }
  *nlevels = n;
  return TANB_OK;
}

int32_t tanb_nu_create(tanb_context* ctx, uint32_t channels, uint32_t ir_length, uint32_t nlevels,
                       const uint32_t* level_block, const uint32_t* level_parts, uint32_t spectrum, tanb_nu** out) {
  if (!ctx || !out || !level_block || !level_parts) return nfail(TANB_INVALID_POINTER, "null argument");
  *out = nullptr;
  if (channels == 0 || ir_length == 0 || nlevels == 0 || nlevels > (uint32_t)tanb::kMaxLevels || spectrum > 2)
    return nfail(TANB_INVALID_ARG, "invalid channels, IR length, level count or spectrum");
  long long off = 0;
  for (uint32_t l = 0; l < nlevels; ++l) {
    const uint32_t N = level_block[l];
    if (N < 32 || N > 8192 || (N & (N - 1)) || level_parts[l] == 0 || (l && N < level_block[l - 1]))
      return nfail(TANB_INVALID_ARG, "level %u: block %u / partitions %u invalid", l, N, level_parts[l]);
    if (l && off < (long long)N)
      return nfail(TANB_INVALID_ARG, "level %u starts at tap %lld < its block %u (would add latency)", l, off, N);
    off += (long long)N * level_parts[l];
  }
  if (off < (long long)ir_length) return nfail(TANB_INVALID_ARG, "levels cover %lld < %u taps", off, ir_length);
  tanb_nu* v = new tanb_nu();
  v->ctx = ctx;
  v->L = (int)ir_length;
  tanb::NuDev& d = v->d;
  d.C = (int)channels;
  d.B0 = (int)level_block[0];
  d.spec = (int)spectrum;
  d.nl = (int)nlevels;
  const size_t Nmax = level_block[nlevels - 1];
  long long omax = 0, o = 0;
  for (uint32_t l = 0; l < nlevels; ++l) {
    omax = std::max(omax, o);
    o += (long long)level_block[l] * level_parts[l];
  }
  d.rin = (int)tanb::pow2_at_least(2 * Nmax + d.B0);
  d.rout = (int)tanb::pow2_at_least((size_t)omax + 2 * Nmax);
  const size_t C = channels;
  const size_t sb = spectrum == 0 ? 8 : 4;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&v->ev_out, cudaEventDisableTiming);
  void* p = nullptr;
  if (e == cudaSuccess && (e = nu_alloc(v, &p, C * d.rin * sizeof(float))) == cudaSuccess) d.in_ring = (float*)p;
  if (e == cudaSuccess && (e = nu_alloc(v, &p, C * d.rout * sizeof(float))) == cudaSuccess) d.out_ring = (float*)p;
  if (e == cudaSuccess && (e = nu_alloc(v, &p, sizeof(long long))) == cudaSuccess) d.k = (long long*)p;
  if (e == cudaSuccess && (e = nu_alloc(v, &p, C * d.B0 * sizeof(float))) == cudaSuccess) v->d_in = (float*)p;
  if (e == cudaSuccess && (e = nu_alloc(v, &p, C * d.B0 * sizeof(float))) == cudaSuccess) v->d_out = (float*)p;
  if (e == cudaSuccess && (e = nu_alloc(v, &p, C * (size_t)ir_length * sizeof(float))) == cudaSuccess)
    v->d_ir = (float*)p;
  o = 0;
  for (uint32_t l = 0; l < nlevels && e == cudaSuccess; ++l) {
    tanb::NuLevel& lv = d.lv[l];
    const size_t N = level_block[l], K = level_parts[l];
    lv.log2N = 0;
    while ((1u << lv.log2N) < N) ++lv.log2N;
    lv.K = (int)K;
    lv.off = o;
    o += (long long)N * K;
    if ((e = nu_alloc(v, &p, C * K * N * sb)) != cudaSuccess) break;
    lv.H = p;
    if (spectrum) {
      if ((e = nu_alloc(v, &p, C * K * sizeof(float))) != cudaSuccess) break;
      lv.scale = (float*)p;
    }
    if ((e = nu_alloc(v, &p, C * K * N * sizeof(float2))) != cudaSuccess) break;
    lv.fdl = (float2*)p;
    if ((e = nu_alloc(v, &p, C * N * sizeof(float2))) != cudaSuccess) break;
    lv.tail = (float2*)p;
    if ((e = nu_alloc(v, &p, 2 * N * sizeof(float2))) != cudaSuccess) break;
    std::vector<float2> tw(2 * N);
    tanb::make_twiddles((int)(2 * N), tw.data());
    // Ordered after this buffer's zero fill, which is queued on the same
    // (non-blocking) stream; a copy on another stream could land first and
    // then be zeroed. A pageable source is staged before the call returns.
    if ((e = cudaMemcpyAsync(p, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, v->stream)) !=
        cudaSuccess)
      break;
    d.tw[l] = (const float2*)p;
  }
  if (e == cudaSuccess) e = cudaMallocHost(&v->h_in, C * d.B0 * sizeof(float));
  if (e == cudaSuccess) e = cudaMallocHost(&v->h_out, C * d.B0 * sizeof(float));
  if (e == cudaSuccess) e = ensure_graphs(v);
  if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
  if (e != cudaSuccess) {
    nu_free(v);
    delete v;
    cudaGetLastError();
    return nfail(e == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "tanb_nu_create: %s",
                 cudaGetErrorString(e));
  }
  std::memset(v->h_in, 0, C * d.B0 * sizeof(float));
  *out = v;
  return TANB_OK;
}

int32_t tanb_nu_release(tanb_nu* v) {
  if (!v) return TANB_OK;
  {
    std::lock_guard<std::mutex> lock(v->mu);
    cudaSetDevice(v->ctx->device);
    nu_free(v);
  }
  delete v;
  return TANB_OK;
}

int32_t tanb_nu_set_response(tanb_nu* v, const float* const* ir, size_t n) {
  if (!v || !ir) return nfail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  if (n > (size_t)v->L) return nfail(TANB_INVALID_ARG, "IR length %zu exceeds %d", n, v->L);
  NU_CUDA(cudaSetDevice(v->ctx->device));
  const tanb::NuDev& d = v->d;
  for (int c = 0; c < d.C; ++c) {
    if (!ir[c] && n) return nfail(TANB_INVALID_ARG, "ppBuffer[%d] == NULL", c);
    if (n)
      NU_CUDA(cudaMemcpyAsync(v->d_ir + (size_t)c * v->L, ir[c], n * sizeof(float), cudaMemcpyHostToDevice,
                              v->stream));
  }
  for (int l = 0; l < d.nl; ++l) NU_CUDA(tanb::launch_nu_ir(d, l, v->d_ir, v->L, (long long)n, v->stream));
  NU_CUDA(cudaStreamSynchronize(v->stream));
  return TANB_OK;
}

int32_t tanb_nu_io(tanb_nu* v, float** in, float** out) {
  if (!v || !in || !out) return nfail(TANB_INVALID_POINTER, "null argument");
  *in = v->h_in;
  *out = v->h_out;
  return TANB_OK;
}

// One base block through the pinned host buffers [C][B0] (one CUDA graph).
int32_t tanb_nu_process(tanb_nu* v) {
  if (!v) return nfail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  NU_CUDA(cudaSetDevice(v->ctx->device));
  const unsigned due = due_mask(v->d, v->k);
  NU_CUDA(ensure_graph(v, due));
  NU_CUDA(cudaGraphLaunch(v->graphs[due], v->stream));
  NU_CUDA(cudaEventSynchronize(v->ev_out));
  v->k += 1;
  return TANB_OK;
}

// One base block with device-resident I/O ([C][ld]); asynchronous.
int32_t tanb_nu_process_device(tanb_nu* v, const float* in, float* out, uint32_t ld) {
  if (!v || !out) return nfail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  NU_CUDA(cudaSetDevice(v->ctx->device));
  NU_CUDA(enqueue_nu_block(v, in, out, ld ? (int)ld : v->d.B0, false, due_mask(v->d, v->k)));
  v->k += 1;
  return TANB_OK;
}

int32_t tanb_nu_synchronize(tanb_nu* v) {
  if (!v) return nfail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  NU_CUDA(cudaSetDevice(v->ctx->device));
  NU_CUDA(cudaStreamSynchronize(v->stream));
  return TANB_OK;
}

void* tanb_nu_stream(tanb_nu* v) { return v ? (void*)v->stream : nullptr; }

int32_t tanb_nu_info(tanb_nu* v, int64_t out[6]) {
  if (!v || !out) return nfail(TANB_INVALID_POINTER, "null argument");
  const tanb::NuDev& d = v->d;
  int64_t bytes_per_block = 0;  // average algorithmic tail bytes per base block
  const int64_t sb = d.spec == 0 ? 8 : 4;
  for (int l = 0; l < d.nl; ++l) {
    const int64_t N = 1LL << d.lv[l].log2N;
    bytes_per_block += (int64_t)d.C * (d.lv[l].K - 1) * N * (8 + sb) * d.B0 / N;
  }
  out[0] = d.C;
  out[1] = d.B0;
  out[2] = d.nl;
  out[3] = (int64_t)v->dev_bytes;
  out[4] = bytes_per_block;
  out[5] = v->k;
  return TANB_OK;
}

}  // extern "C"
