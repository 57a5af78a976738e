// Shared-memory Stockham FFT and the real-FFT packing used by every kernel.
//
// A 2M-point real transform runs as an M-point complex transform of
// z[n] = v[2n] + i v[2n+1], followed by the standard split step
//   X[k] = 1/2 (Z[k] + Z*[M-k]) - i/2 W^k (Z[k] - Z*[M-k]),   W = exp(-2 pi i / 2M)
// and the inverse runs the mirror step before an M-point inverse transform.
// Spectra are packed: bin 0 holds (X[0], X[M]), both real.
//
// The complex transform is a radix-4 Stockham autosort FFT (one radix-2 stage
// first when log2 M is odd), in place in shared memory: every thread loads its
// butterflies' inputs into registers, the block synchronises, and the outputs
// go back to the autosorted positions. Twiddles come from a table of W^j,
// j in [0, 2M), computed in double on the host and rounded to float.
#pragma once

#include <cuda_runtime.h>

namespace tanb {

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }

// Threads per FFT block and complex values each thread holds per stage.
// TW_SMEM: the 2M-entry twiddle table is staged in shared memory (it fits
// beside two M-point work buffers up to M = 2048).
template <int LOG2M>
struct FftShape {
  static constexpr int M = 1 << LOG2M;
  static constexpr int T = (M / 4 > 1024) ? 1024 : M / 4;
  static constexpr int E = M / T;
  static constexpr bool TW_SMEM = LOG2M <= 11;
  // bin pairs (k, M-k), k in [0, M/2], handled per thread
  static constexpr int KP = (M / 2 + 1 + T - 1) / T;
};

// In-place M-point complex FFT of s[0..M) (forward: exp(-i..), inverse:
// exp(+i..), unscaled). `tw` may point to global or shared memory. Must be
// called by all FftShape<LOG2M>::T threads; ends with a barrier.
template <int LOG2M, bool INV>
__device__ __forceinline__ void fft_inplace(float2* s, const float2* __restrict__ tw) {
  using S = FftShape<LOG2M>;
  constexpr int M = S::M, T = S::T, E = S::E, N = 2 * M;
  const int tid = threadIdx.x;
  int Ns = 1;
  if constexpr ((LOG2M & 1) != 0) {
    constexpr int nb = M / 2;
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const int j = tid + e * T;
      v[2 * e] = s[j];
      v[2 * e + 1] = s[j + nb];
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const int j = tid + e * T;
      s[2 * j] = c_add(v[2 * e], v[2 * e + 1]);
      s[2 * j + 1] = c_sub(v[2 * e], v[2 * e + 1]);
    }
    __syncthreads();
    Ns = 2;
  }
#pragma unroll 1
  for (; Ns < M; Ns <<= 2) {
    constexpr int nb = M / 4;
    const int tstep = N / (4 * Ns);
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E / 4; ++e) {
      const int j = tid + e * T;
      const int k = j & (Ns - 1);
      v[4 * e] = s[j];
#pragma unroll
      for (int r = 1; r < 4; ++r) {
        float2 w = tw[r * k * tstep];
        if (INV) w.y = -w.y;
        v[4 * e + r] = c_mul(s[j + r * nb], w);
      }
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E / 4; ++e) {
      const int j = tid + e * T;
      const int k = j & (Ns - 1);
      const float2 t0 = c_add(v[4 * e], v[4 * e + 2]);
      const float2 t1 = c_sub(v[4 * e], v[4 * e + 2]);
      const float2 t2 = c_add(v[4 * e + 1], v[4 * e + 3]);
      const float2 t3 = c_sub(v[4 * e + 1], v[4 * e + 3]);
      // forward: X1 = t1 - i t3, X3 = t1 + i t3; inverse: swapped
      const float2 it3 = make_float2(-t3.y, t3.x);
      const int d = ((j - k) << 2) + k;
      s[d] = c_add(t0, t2);
      s[d + Ns] = INV ? c_add(t1, it3) : c_sub(t1, it3);
      s[d + 2 * Ns] = c_sub(t0, t2);
      s[d + 3 * Ns] = INV ? c_sub(t1, it3) : c_add(t1, it3);
    }
    __syncthreads();
  }
}

// Split step of the forward real transform for bin k (a = Z[k], b = Z[M-k],
// w = W^k): returns X[k].
__device__ __forceinline__ float2 rfft_post(float2 a, float2 b, float2 w) {
  const float2 bc = c_conj(b);
  const float2 e = make_float2(0.5f * (a.x + bc.x), 0.5f * (a.y + bc.y));
  const float2 d = make_float2(0.5f * (a.x - bc.x), 0.5f * (a.y - bc.y));
  const float2 t = c_mul(w, d);
  return make_float2(e.x + t.y, e.y - t.x);
}

// Mirror step of the inverse real transform for bin k (a = A[k],
// b = A[M-k], w = W^k), scaled by inv_n = 1/2M: returns Z'[k].
__device__ __forceinline__ float2 irfft_pre(float2 a, float2 b, float2 w, float inv_n) {
  const float2 bc = c_conj(b);
  const float2 e = c_add(a, bc);
  const float2 d = c_sub(a, bc);
  const float2 o = c_mul(d, c_conj(w));
  return make_float2((e.x - o.y) * inv_n, (e.y + o.x) * inv_n);
}

// Packed bin 0: forward (Z[0] -> (X[0], X[M])) and inverse.
__device__ __forceinline__ float2 rfft_post_dc(float2 z0) { return make_float2(z0.x + z0.y, z0.x - z0.y); }
__device__ __forceinline__ float2 irfft_pre_dc(float2 a, float inv_n) {
  return make_float2((a.x + a.y) * inv_n, (a.x - a.y) * inv_n);
}

// acc + a * b with the operation order of the reference's AVX2 planar MAC
// (re: fma(ar, br, -(ai*bi)) + cr, im: fma(ar, bi, ai*br) + ci).
__device__ __forceinline__ float2 c_mac(float2 acc, float2 a, float2 b) {
  const float re = __fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y));
  const float im = __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x));
  return make_float2(__fadd_rn(re, acc.x), __fadd_rn(im, acc.y));
}
// Packed bin 0: two independent real products.
__device__ __forceinline__ float2 c_mac_dc(float2 acc, float2 a, float2 b) {
  return make_float2(__fadd_rn(__fmul_rn(a.x, b.x), acc.x), __fadd_rn(__fmul_rn(a.y, b.y), acc.y));
}

}  // namespace tanb
