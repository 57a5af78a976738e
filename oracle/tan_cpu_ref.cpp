// TEST INFRASTRUCTURE ONLY -- the oracle. Nothing in the product (libtanb.so,
// the tan_b200 package) links, loads or calls this file; only tests/, the
// smoke check and bench.py's CPU-baseline / reference legs do, as the checker.
//
// A CPU restatement of AMD TrueAudio Next's uniformly-partitioned FFT
// convolution (TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM on the CPU):
//
//   layout      planar real-FFT partitions of stride S = 2B + 16 floats,
//               re plane at [0, B+8), im plane at [B+8, 2B+16)
//               (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.h:50,
//                ConvolutionImpl.cpp:1548-1663)
//   IR prep     split the time-domain IR into P = nextpow2(L)/B partitions,
//               zero-pad each to 2B and R2C-transform it
//               (ConvolutionImpl.cpp:2080-2141)
//   head        newest FDL slot <- R2C([x_k, 0^B]); acc += X_k * H_0;
//               C2R (scaled 1/N); y = acc[0..B) + overlap; overlap <- acc[B..2B)
//               (ConvolutionImpl.cpp:2380-2535)
//   tail        acc_next = sum_{i=1}^{P-1} FDL[(cur+i-1) mod P] * H_i
//               (ConvolutionImpl.cpp:2539-2643)
//   MAC         cr += fmsub(ar, br, ai*bi); ci += fmadd(ar, bi, ai*br) on
//               8-wide planar vectors, count B+8, OpenMP over channels
//               (tan/tanlibrary/src/TrueAudioNext/math/MathImpl.cpp:495-530)
//   C2R scale   1/N (tan/tanlibrary/src/TrueAudioNext/fft/FFTImpl.cpp:1046-1051)
//   crossfade   out = new*(j/F) + old*((F-j)/F), F = B
//               (ConvolutionImpl.cpp:877, 1392-1408)
//   flags       STOP_INPUT ring-out of nextpow2(L) samples then flush,
//               FLUSH_STREAM, free-channel query
//               (ConvolutionImpl.cpp:2867-2907, 1084-1110)
//
// Differences from the reference, all deliberate:
//  * The FFT is our own (radix-2, twiddles computed in double and rounded to
//    float): the reference dlopens FFTW 3.3.5, which is absent here.
//  * IR activation is deterministic: the new IR takes effect on the first
//    block processed after UpdateResponseTD returns (the reference hands it to
//    a background thread, so the swap block depends on thread timing).
//  * The swap block computes the new IR's output over the full input history
//    (its own tail and overlap) and blends it with the old IR's output; the
//    reference runs ProcessInternal twice with time advancing twice
//    (ConvolutionImpl.cpp:976-990), which corrupts the delay line.
//  * Per-channel state is indexed by channel, not by running-channel rank, and
//    a flush also clears the precomputed tail (the reference's CPU flush
//    dereferences an unallocated state array, ConvolutionImpl.cpp:1284-1325).
//  * A free channel (rung out or stopped+flushed) that runs again starts from
//    silence; the reference keeps whatever its last ring-out block left.
#include <immintrin.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

enum : int32_t {
  kOk = 0,
  kInvalidArg = 4,
  kNotSupported = 10,
  kNotFound = 11,
  kNotInitialized = 13,
  kWrongState = 15,
};
constexpr uint32_t kStopInput = 1;
constexpr uint32_t kFlushStream = 2;
constexpr int kPad = 16;  // PARTITION_PAD_FFTREAL_PLANAR

// Real FFT of size N = 2M through a complex FFT of size M (even/odd packing).
// Planar spectrum: re[0..M], im[0..M] (M+1 bins).
struct RealFFT {
  int N = 0, M = 0, logM = 0;
  std::vector<float> wr, wi;   // W_N^j = exp(-2 pi i j / N), j in [0, N)
  std::vector<int> rev;        // bit reversal over M points
  std::vector<float> zr, zi;   // scratch, per thread

  void init(int n) {
    N = n;
    M = n / 2;
    logM = 0;
    while ((1 << logM) < M) ++logM;
    wr.resize(N);
    wi.resize(N);
    for (int j = 0; j < N; ++j) {
      double a = -2.0 * M_PI * (double)j / (double)N;
      wr[j] = (float)std::cos(a);
      wi[j] = (float)std::sin(a);
    }
    rev.resize(M);
    for (int i = 0; i < M; ++i) {
      int r = 0;
      for (int b = 0; b < logM; ++b) r |= ((i >> b) & 1) << (logM - 1 - b);
      rev[i] = r;
    }
  }

  // In-place radix-2 decimation-in-time FFT of size M on (re, im) that are
  // already in bit-reversed order. sign = -1 forward, +1 inverse (unscaled).
  void cfft(float* re, float* im, int sign) const {
    for (int len = 2; len <= M; len <<= 1) {
      int half = len >> 1;
      int tstep = (N / len);  // W_len^k = W_N^(k * N/len)
      for (int s = 0; s < M; s += len) {
        for (int k = 0; k < half; ++k) {
          float c = wr[k * tstep];
          float d = sign < 0 ? wi[k * tstep] : -wi[k * tstep];
          int a = s + k, b = a + half;
          float tr = re[b] * c - im[b] * d;
          float ti = re[b] * d + im[b] * c;
          re[b] = re[a] - tr;
          im[b] = im[a] - ti;
          re[a] = re[a] + tr;
          im[a] = im[a] + ti;
        }
      }
    }
  }

  // x: N reals -> re[0..M], im[0..M]
  void forward(const float* x, float* re, float* im, float* zr_, float* zi_) const {
    for (int n = 0; n < M; ++n) {
      int r = rev[n];
      zr_[r] = x[2 * n];
      zi_[r] = x[2 * n + 1];
    }
    cfft(zr_, zi_, -1);
    // X[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 W_N^k (Z[k] - conj Z[M-k])
    re[0] = zr_[0] + zi_[0];
    im[0] = 0.f;
    re[M] = zr_[0] - zi_[0];
    im[M] = 0.f;
    for (int k = 1; k < M; ++k) {
      float ar = zr_[k], ai = zi_[k];
      float br = zr_[M - k], bi = -zi_[M - k];  // conj Z[M-k]
      float er = 0.5f * (ar + br), ei = 0.5f * (ai + bi);
      float dr = 0.5f * (ar - br), di = 0.5f * (ai - bi);
      // -i * W * d
      float wrk = wr[k], wik = wi[k];
      float tr = wrk * dr - wik * di;
      float ti = wrk * di + wik * dr;
      re[k] = er + ti;
      im[k] = ei - tr;
    }
  }

  // re[0..M], im[0..M] -> y: N reals, scaled by 1/N
  void inverse(const float* re, const float* im, float* y, float* zr_, float* zi_) const {
    const float scale = 1.0f / (float)N;
    for (int k = 0; k < M; ++k) {
      float ar = re[k], ai = (k == 0) ? 0.f : im[k];
      float br = re[M - k], bi = (k == 0) ? 0.f : -im[M - k];  // conj A[M-k]
      if (k == 0) { br = re[M]; bi = 0.f; }
      float er = ar + br, ei = ai + bi;         // 2 X_e
      float dr = ar - br, di = ai - bi;         // 2 X_o W^k
      // X_o = d * W_N^{-k} = d * conj(W_N^k)
      float wrk = wr[k], wik = -wi[k];
      float orr = dr * wrk - di * wik;
      float oi = dr * wik + di * wrk;
      // Z = X_e + i X_o
      int r = rev[k];
      zr_[r] = (er - oi) * scale;
      zi_[r] = (ei + orr) * scale;
    }
    cfft(zr_, zi_, +1);
    for (int n = 0; n < M; ++n) {
      y[2 * n] = zr_[n];
      y[2 * n + 1] = zi_[n];
    }
  }
};

// Planar complex multiply-accumulate, 8 lanes at a time, same operation order
// as TANMathImpl::PlanarComplexMultiplyAccumulate's AVX2 branch.
inline void planar_cmac(const float* a, const float* b, float* acc, int count, int spacing) {
  for (int k = 0; k < count; k += 8) {
    __m256 ar = _mm256_loadu_ps(a + k);
    __m256 ai = _mm256_loadu_ps(a + spacing + k);
    __m256 br = _mm256_loadu_ps(b + k);
    __m256 bi = _mm256_loadu_ps(b + spacing + k);
    __m256 cr = _mm256_loadu_ps(acc + k);
    __m256 ci = _mm256_loadu_ps(acc + spacing + k);
    cr = _mm256_add_ps(_mm256_fmsub_ps(ar, br, _mm256_mul_ps(ai, bi)), cr);
    ci = _mm256_add_ps(_mm256_fmadd_ps(ar, bi, _mm256_mul_ps(ai, br)), ci);
    _mm256_storeu_ps(acc + k, cr);
    _mm256_storeu_ps(acc + spacing + k, ci);
  }
}

struct RefConv {
  int L = 0, B = 0, C = 0, P = 0, S = 0, N = 0, length = 0, threads = 1;
  RealFFT fft;
  // IR spectra: [slot 0/1][channel] -> P*S floats
  std::vector<float> H[2];
  std::vector<int> active;       // per channel: active slot
  std::vector<uint8_t> pending;  // per channel: new IR waiting in 1-active
  std::vector<float> fdl;        // [channel] -> P*S floats (frequency-domain delay line)
  std::vector<float> overlap;    // [channel] -> B
  std::vector<float> tail;       // [channel] -> S (precomputed tail for the next block)
  std::vector<float> work;       // per thread scratch: several S-sized buffers
  int cur = 0;                   // newest FDL slot
  // channel-flag state
  std::vector<int> tailLeft;
  std::vector<uint8_t> available, flushed;

  float* h(int slot, int c) { return H[slot].data() + (size_t)c * P * S; }
  float* fdlc(int c) { return fdl.data() + (size_t)c * P * S; }

  void flush(int c) {
    std::memset(fdlc(c), 0, sizeof(float) * (size_t)P * S);
    std::memset(overlap.data() + (size_t)c * B, 0, sizeof(float) * B);
    std::memset(tail.data() + (size_t)c * S, 0, sizeof(float) * S);
  }

  // sum_{i=i0}^{P-1} FDL[(base + i) mod P] * Hslot_i  into acc (S floats, zeroed first)
  void fdl_mac(int c, const float* hs, int base, int i0, float* acc) {
    std::memset(acc, 0, sizeof(float) * S);
    for (int i = i0; i < P; ++i) {
      int slot = ((base + i) % P + P) % P;
      planar_cmac(fdlc(c) + (size_t)slot * S, hs + (size_t)i * S, acc, B + 8, B + 8);
    }
  }
};

}  // namespace

extern "C" {

void* tanref_create(int L, int B, int C, int threads) {
  if (L <= 0 || B <= 0 || C <= 0 || (B & (B - 1)) != 0 || B < 8) return nullptr;
  RefConv* r = new RefConv();
  r->L = L;
  r->B = B;
  r->C = C;
  r->threads = threads > 0 ? threads : 1;
  int len = 1;
  while (len < L) len <<= 1;
  r->length = len;
  r->P = len / B;
  if (r->P < 1) r->P = 1;
  r->S = 2 * B + kPad;
  r->N = 2 * B;
  r->fft.init(r->N);
  size_t per = (size_t)r->P * r->S;
  r->H[0].assign(per * C, 0.f);
  r->H[1].assign(per * C, 0.f);
  r->active.assign(C, 0);
  r->pending.assign(C, 0);
  r->fdl.assign(per * C, 0.f);
  r->overlap.assign((size_t)B * C, 0.f);
  r->tail.assign((size_t)r->S * C, 0.f);
  r->work.assign((size_t)r->threads * 8 * r->S, 0.f);
  r->cur = 0;
  r->tailLeft.assign(C, 0);
  r->available.assign(C, 0);
  r->flushed.assign(C, 0);
  return r;
}

void tanref_destroy(void* h) { delete static_cast<RefConv*>(h); }

int tanref_partitions(void* h) { return static_cast<RefConv*>(h)->P; }

// UpdateResponseTD (ConvolutionImpl.cpp:407-557 + the update thread's
// partition/transform, :2080-2141), done synchronously.
int tanref_update_td(void* hh, const float* const* ir, size_t n, const uint32_t* flags) {
  RefConv* r = static_cast<RefConv*>(hh);
  if (!ir) return kInvalidArg;
  if (n > (size_t)r->L) return kInvalidArg;
  for (int c = 0; c < r->C; ++c)
    if (flags && (flags[c] & kFlushStream)) r->flush(c);
  // one forward transform per partition per channel, OpenMP over channels as
  // in TANFFTImpl::TransformImplCpuOMP (FFTImpl.cpp:1091-1096)
#pragma omp parallel for num_threads(r->threads) schedule(static)
  for (int c = 0; c < r->C; ++c) {
    if (flags && (flags[c] & kStopInput)) continue;
    int slot = 1 - r->active[c];
    float* hs = r->h(slot, c);
    std::vector<float> td((size_t)r->P * r->B + r->B, 0.f);
    std::memcpy(td.data(), ir[c], sizeof(float) * n);
    std::vector<float> frame(r->N), zr(r->B), zi(r->B);
    for (int i = 0; i < r->P; ++i) {
      std::fill(frame.begin(), frame.end(), 0.f);
      std::memcpy(frame.data(), td.data() + (size_t)i * r->B, sizeof(float) * r->B);
      float* part = hs + (size_t)i * r->S;
      std::memset(part, 0, sizeof(float) * r->S);
      r->fft.forward(frame.data(), part, part + r->B + 8, zr.data(), zi.data());
    }
    r->pending[c] = 1;
  }
  return kOk;
}

// Process(float**, float**, ...) for FFT_PARTITIONED_UNIFORM on the CPU:
// state machine (ConvolutionImpl.cpp:848-1043), ProcessInternal's channel
// flags (:2839-2931), head (:2380-2535) and tail (:2539-2643).
int tanref_process(void* hh, const float* const* in, float* const* out, size_t n,
                   const uint32_t* flags, size_t* done) {
  RefConv* r = static_cast<RefConv*>(hh);
  if (!in || !out) return kInvalidArg;
  if (done) *done = 0;
  const int B = r->B, S = r->S, P = r->P, C = r->C;
  size_t nblocks = n / (size_t)B;
  for (size_t blk = 0; blk < nblocks; ++blk) {
    // channel flags
    std::vector<uint8_t> run(C, 0);
    int nrun = 0;
    for (int c = 0; c < C; ++c) {
      uint32_t f = flags ? flags[c] : 0u;
      const bool was_free = r->available[c] != 0;
      if (!flags) {
        r->available[c] = 0;
        r->tailLeft[c] = r->length;
      } else if (f & kStopInput) {
        if (f & kFlushStream) {
          r->available[c] = 1;
          r->tailLeft[c] = 0;
        } else if (r->tailLeft[c] > 0) {
          r->available[c] = 0;
          r->tailLeft[c] -= B;
          if (r->tailLeft[c] <= 0) r->flush(c);
        } else {
          r->available[c] = 1;
          r->tailLeft[c] = 0;
        }
      } else {
        r->available[c] = 0;
        r->tailLeft[c] = r->length;
      }
      if (flags && (f & kFlushStream)) {
        if (!r->flushed[c]) r->flush(c);
        r->flushed[c] = 1;
      } else {
        r->flushed[c] = 0;
      }
      run[c] = !r->available[c];
      // a free channel that starts running again starts from silence
      if (was_free && run[c]) r->flush(c);
      nrun += run[c];
    }
    if (nrun == 0) return kWrongState;

    const int prev = r->cur;               // newest slot before this block
    const int cur = (prev - 1 + P) % P;    // slot for this block's spectrum
    r->cur = cur;

#pragma omp parallel for num_threads(r->threads) schedule(static)
    for (int c = 0; c < C; ++c) {
      if (!run[c]) continue;
      int t = omp_get_thread_num();
      float* w = r->work.data() + (size_t)t * 8 * S;
      float* accA = w;            // old / only IR accumulator
      float* accB = w + S;        // new IR accumulator (swap block)
      float* ovlN = w + 2 * S;    // new IR overlap (swap block)
      float* tA = w + 3 * S;      // time-domain scratch (2B)
      float* tB = w + 4 * S;
      float* zr = w + 5 * S;
      float* zi = w + 6 * S;
      const float* x = in[c] + blk * B;
      float* y = out[c] + blk * B;
      const bool swap = r->pending[c] != 0;
      const float* hOld = r->h(r->active[c], c);
      const float* hNew = r->h(1 - r->active[c], c);

      if (swap) {
        // New IR's overlap: upper half of C2R(sum_{i=0}^{P-1} X_{k-1-i} H'_i),
        // and new IR's tail for this block, both from the delay line before
        // this block's spectrum is inserted.
        r->fdl_mac(c, hNew, prev, 0, accB);
        r->fft.inverse(accB, accB + B + 8, tB, zr, zi);
        std::memcpy(ovlN, tB + B, sizeof(float) * B);
        r->fdl_mac(c, hNew, prev - 1, 1, accB);
      }

      // newest slot <- R2C([x_k, 0^B])
      float* part = r->fdlc(c) + (size_t)cur * S;
      std::memset(tA, 0, sizeof(float) * 2 * B);
      std::memcpy(tA, x, sizeof(float) * B);
      std::memset(part, 0, sizeof(float) * S);
      r->fft.forward(tA, part, part + B + 8, zr, zi);

      // head: acc = tail + X_k * H_0
      std::memcpy(accA, r->tail.data() + (size_t)c * S, sizeof(float) * S);
      planar_cmac(part, hOld, accA, B + 8, B + 8);
      r->fft.inverse(accA, accA + B + 8, tA, zr, zi);
      float* ovl = r->overlap.data() + (size_t)c * B;
      if (!swap) {
        for (int i = 0; i < B; ++i) y[i] = tA[i] + ovl[i];
        std::memcpy(ovl, tA + B, sizeof(float) * B);
      } else {
        planar_cmac(part, hNew, accB, B + 8, B + 8);
        r->fft.inverse(accB, accB + B + 8, tB, zr, zi);
        const float step = 1.0f / (float)B;
        for (int i = 0; i < B; ++i) {
          float yo = tA[i] + ovl[i];
          float yn = tB[i] + ovlN[i];
          float w1 = step * (float)i;
          float w2 = step * (float)(B - i);
          y[i] = yn * w1 + yo * w2;
        }
        std::memcpy(ovl, tB + B, sizeof(float) * B);
        r->active[c] = 1 - r->active[c];
        r->pending[c] = 0;
      }
      // tail for the next block: sum_{i=1}^{P-1} FDL[(cur+i-1) mod P] * H_i
      r->fdl_mac(c, r->h(r->active[c], c), cur - 1, 1, r->tail.data() + (size_t)c * S);
    }
    if (done) *done += B;
  }
  return kOk;
}

// GetNextFreeChannel (ConvolutionImpl.cpp:1084-1110)
int tanref_next_free_channel(void* hh, uint32_t* idx, const uint32_t* flags) {
  RefConv* r = static_cast<RefConv*>(hh);
  if (!idx) return kInvalidArg;
  *idx = 0xFFFFFFFFu;
  if (!flags) return kNotFound;
  for (int c = 0; c < r->C; ++c) {
    if ((flags[c] & kStopInput) && r->tailLeft[c] <= 0) {
      *idx = (uint32_t)c;
      return kOk;
    }
  }
  return kNotFound;
}

// TIME_DOMAIN method: ProcessDirect (ConvolutionImpl.cpp:721-762) over
// ovlTimeDomainCPU (:2757-2782). One circular history of nextpow2(L) samples
// per channel; each call appends n <= nextpow2(L) samples and computes
//   out[j] = sum_{k=first}^{last-1} hist[(pos + j - k) mod len] * ir[k]
// accumulating in float in increasing k.
struct RefTD {
  int L = 0, C = 0, length = 0;
  std::vector<float> hist;  // [C][length]
  std::vector<int> pos;     // per channel
};

void* tanref_td_create(int L, int C) {
  if (L <= 0 || C <= 0) return nullptr;
  RefTD* r = new RefTD();
  r->L = L;
  r->C = C;
  int len = 1;
  while (len < L) len <<= 1;
  r->length = len;
  r->hist.assign((size_t)C * len, 0.f);
  r->pos.assign(C, 0);
  return r;
}

void tanref_td_destroy(void* h) { delete static_cast<RefTD*>(h); }

int tanref_td_process_direct(void* hh, const float* const* ir, const float* const* in, float* const* out,
                             size_t n, size_t* done, const int* nz) {
  RefTD* r = static_cast<RefTD*>(hh);
  const int len = r->length;
  if (n > (size_t)len) n = len;
  for (int c = 0; c < r->C; ++c) {
    int first = 0, last = len;
    if (nz) {
      first = nz[2 * c];
      last = nz[2 * c + 1];
    }
    float* hist = r->hist.data() + (size_t)c * len;
    const int p = r->pos[c] % len;
    for (size_t i = 0; i < n; ++i) hist[(p + i) % len] = in[c][i];
    for (size_t j = 0; j < n; ++j) {
      float acc = 0.f;
      for (int k = first; k < last; ++k) acc += hist[((size_t)p + j - k + len) % len] * ir[c][k];
      out[c][j] = acc;
    }
    r->pos[c] += (int)n;
  }
  if (done) *done = n;
  return kOk;
}

// Plain forward/inverse real FFT, exposed for the oracle's own tests.
int tanref_rfft(int N, const float* x, float* re, float* im) {
  RealFFT f;
  f.init(N);
  std::vector<float> zr(N / 2), zi(N / 2);
  f.forward(x, re, im, zr.data(), zi.data());
  return kOk;
}

int tanref_irfft(int N, const float* re, const float* im, float* y) {
  RealFFT f;
  f.init(N);
  std::vector<float> zr(N / 2), zi(N / 2);
  f.inverse(re, im, y, zr.data(), zi.data());
  return kOk;
}

// ---------------------------------------------------------------------------
// TANConverter and TANMixer (test infrastructure, as everything in this file).
// ---------------------------------------------------------------------------

// short -> float, TANConverterImpl::Convert(short*, ...) ConverterImpl.cpp:217-246:
// out = (float)in * (gain / SHRT_MAX), scale rounded once to float.
void tanref_convert_s16_f32(const int16_t* in, size_t in_step, size_t n, float* out, size_t out_step, float gain) {
  const float scale = gain / 32767;
  for (size_t i = 0; i < n; ++i) out[i * out_step] = in[i * in_step] * scale;
}

// float -> short, TANConverterImpl::Convert(float*, ...) ConverterImpl.cpp:287-408
// with its SSE2 path taken (ConverterImpl.cpp:69): while at least 8 samples
// remain, 8 products are rounded to nearest even by cvtps2dq (out-of-range and
// NaN give INT_MIN) and packed to 16 bits with saturation, without setting
// the clip flag; the last n mod 8 samples are truncated toward zero (cvttss2si,
// INT_MIN out of range), clamped, and set the flag when clamped.
void tanref_convert_f32_s16(const float* in, size_t in_step, size_t n, int16_t* out, size_t out_step, float gain,
                            int32_t* clipped) {
  const float scale = 32767 * gain;
  bool clip = false;
  size_t i = 0;
  for (; n - i >= 8; i += 8) {
    alignas(16) float f[8];
    for (int j = 0; j < 8; ++j) f[j] = in[(i + j) * in_step] * scale;
    const __m128i a = _mm_cvtps_epi32(_mm_load_ps(f));
    const __m128i b = _mm_cvtps_epi32(_mm_load_ps(f + 4));
    alignas(16) int16_t s8[8];
    _mm_store_si128(reinterpret_cast<__m128i*>(s8), _mm_packs_epi32(a, b));
    for (int j = 0; j < 8; ++j) out[(i + j) * out_step] = s8[j];
  }
  for (; i < n; ++i) {
    const float f = in[i * in_step] * scale;
    long v = _mm_cvttss_si32(_mm_set_ss(f));
    if (v > 32767) {
      v = 32767;
      clip = true;
    }
    if (v < -32768) {
      v = -32768;
      clip = true;
    }
    out[i * out_step] = (int16_t)v;
  }
  if (clipped) *clipped = clip ? 1 : 0;
}

// float -> short as the reference's OpenCL kernel floatToShort
// (Converter.cl:97-120): clamp to [SHRT_MIN, SHRT_MAX] setting the flag, then
// convert_short (round toward zero). NaN converts to 0 here (the kernel leaves
// it to the device).
void tanref_convert_f32_s16_dev(const float* in, size_t in_step, size_t n, int16_t* out, size_t out_step, float gain,
                                int32_t* clipped) {
  const float scale = 32767 * gain;
  bool clip = false;
  for (size_t i = 0; i < n; ++i) {
    float f = in[i * in_step] * scale;
    if (f > 32767) {
      f = 32767;
      clip = true;
    }
    if (f < -32768) {
      f = -32768;
      clip = true;
    }
    out[i * out_step] = (f != f) ? 0 : (int16_t)f;
  }
  if (clipped) *clipped = clip ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Room response producer: the GPU path of TrueAudioVR::generateRoomResponse
// (samples/src/TrueAudioVR/TrueAudioVR.cpp:659-786 with GENROOM_USE_GPU_MEM;
// kernels Kernels/GenerateRoomResponse.cl:206-321 and Kernels/Fill.cl).
// Differences from the reference, all deliberate: damp^k for the integer wall
// counts k by repeated multiplication (the kernel's native_powr is
// implementation-defined), sqrt correctly rounded (native_sqrt), sums in 64
// bits (the kernel's int32 can wrap) converted as signed (Fill.cl converts
// them as unsigned, which turns negative sums into large positive values).
// ---------------------------------------------------------------------------
static float pow_int(float b, int k) {
  float r = 1.0f;
  for (int i = 0; i < k; ++i) r = r * b;
  return r;
}

// One ear: the kernel's per-image work over its grid. Returns the image count.
static long room_ear(const float* room, const float* src, float hx, float hy, float hz, float evx, float evy, float evz,
                     float earV, float maxGain, float dMin, int rate, int length, int hrtfLength, int filterLength,
                     const float* lpF, const float* hpF, int numRefX, int numRefY, int numRefZ, int64_t* acc) {
  const float W = room[0], H = room[1], L = room[2];
  const float dRight = room[4], dLeft = room[3], dTop = room[5], dBottom = room[6], dFront = room[7],
              dBack = room[8];
  const float kF2I = 67108864.0f;
  auto up4 = [](int n) { return (n % 4) ? n + 4 - n % 4 : n; };  // the NDRange rounding (local size 4)
  const int gx = up4(numRefX), gy = up4(numRefY), gz = up4(numRefZ);
  long images = 0;
  for (int z = 0; z < gz && z <= numRefZ; ++z)
    for (int y = 0; y < gy && y <= numRefY; ++y)
      for (int x = 0; x < gx && x <= numRefX; ++x) {
        ++images;
        const int ix = x - numRefX / 2, iy = y - numRefY / 2, iz = z - numRefZ / 2;
        float a = (ix % 2 == 0) ? (float)ix : (float)(ix + 1);
        float b = (ix % 2 == 0) ? 1.0f : -1.0f;
        const float rx = a * W + b * src[0];
        a = (iy % 2 == 0) ? (float)iy : (float)(iy + 1);
        b = (iy % 2 == 0) ? 1.0f : -1.0f;
        const float ry = a * H + b * src[1];
        a = (iz % 2 == 0) ? (float)iz : (float)(iz + 1);
        b = (iz % 2 == 0) ? 1.0f : -1.0f;
        const float rz = a * L + b * src[2];
        const int kxl = ix > 0 ? ix / 2 : std::abs(ix - 1) / 2, kyb = iy > 0 ? iy / 2 : std::abs(iy - 1) / 2,
                  kzb = iz > 0 ? iz / 2 : std::abs(iz - 1) / 2;
        const int kxr = ix > 0 ? (ix + 1) / 2 : std::abs(ix) / 2, kyt = iy > 0 ? (iy + 1) / 2 : std::abs(iy) / 2,
                  kzf = iz > 0 ? (iz + 1) / 2 : std::abs(iz) / 2;
        float amp = pow_int(dRight, kxr);
        amp = amp * pow_int(dLeft, kxl);
        amp = amp * pow_int(dTop, kyt);
        amp = amp * pow_int(dBottom, kyb);
        amp = amp * pow_int(dFront, kzf);
        amp = amp * pow_int(dBack, kzb);
        const float dx = rx - hx, dy = ry - hy, dz = rz - hz;
        const float d = std::sqrt(dx * dx + dy * dy + dz * dz);
        const int fi = 1 + (int)((d / 340.0f) * (float)rate);
        if (fi >= length) continue;
        const float dr = (d <= dMin) ? maxGain : maxGain * dMin / d;
        const int len = std::min(filterLength, length - fi);
        const float dp = evx * dx + evy * dy + evz * dz;
        const float cosA = dp / (earV * d);
        const float hf = (cosA + 1.0f) / 2.0f;
        if (fi < hrtfLength) {
          for (int i = 0; i < len; ++i) acc[fi + i] += (int64_t)(int32_t)(kF2I * amp * dr * (lpF[i] + hf * hpF[i]));
        } else {
          acc[fi] += (int64_t)(int32_t)(kF2I * amp * dr);
        }
      }
  return images;
}

// room[9]: width, height, length, damp left, right, top, bottom, front, back.
// src[3]; ears[7]: head x, y, z, ear spacing, yaw, pitch, roll (degrees).
// Returns the number of images per ear (-1: invalid room).
long tanref_room_response(const float* room_in, const float* src_in, const float* ears, int rate, int length,
                          int filterLength, const float* lowPass, const float* highPass, int flags, int maxBounces,
                          float* left, float* right) {
  float room[9];
  std::memcpy(room, room_in, sizeof(room));
  float src[3] = {src_in[0], src_in[1], src_in[2]};
  // TrueAudioVR.cpp:663-668: source clamped into the room
  src[0] = std::min(std::max(src[0], 0.0f), room[0]);
  src[1] = std::min(std::max(src[1], 0.0f), room[1]);
  src[2] = std::min(std::max(src[2], 0.0f), room[2]);
  // :670-689 ear offsets and orientation vectors, rotated by yaw / pitch / roll
  const float es = ears[3];
  // left / right ear offsets, then left / right ear vectors (earVzL = -earDxL, earVzR = earDxR)
  float e[4][3] = {{es / 2, 0.0f, 0.0f}, {-es / 2, 0.0f, 0.0f}, {es / 2, 0.0f, -(es / 2)}, {-es / 2, 0.0f, -es / 2}};
  const float pi = (float)3.141592653589793;
  const float sY = std::sin(ears[4] * pi / 180), cY = std::cos(ears[4] * pi / 180);
  const float sP = std::sin(ears[5] * pi / 180), cP = std::cos(ears[5] * pi / 180);
  const float sR = std::sin(ears[6] * pi / 180), cR = std::cos(ears[6] * pi / 180);
  const float m[3][3] = {{cR * cY - sR * sP * sY, -sR * cP, cR * sY + sR * sP * cY},
                         {sR * cY + cR * sP * sY, cR * cP, sR * sY - cR * sP * cY},
                         {-cP * sY, sP, cP * cY}};
  for (auto& v : e) {
    const float x = v[0], y = v[1], z = v[2];
    v[0] = x * m[0][0] + y * m[0][1] + z * m[0][2];
    v[1] = x * m[1][0] + y * m[1][1] + z * m[1][2];
    v[2] = x * m[2][0] + y * m[2][1] + z * m[2][2];
  }
  const int nSW = (int)((room[0] / 340.0f) * rate), nSH = (int)((room[1] / 340.0f) * rate),
            nSL = (int)((room[2] / 340.0f) * rate);
  if (nSW <= 0 || nSH <= 0 || nSL <= 0) return -1;
  int nW = 1 + length / nSW, nH = 1 + length / nSH, nL = 1 + length / nSL;
  if (flags & 0x40) {  // GENROOM_LIMIT_BOUNCES
    nW = std::min(nW, maxBounces);
    nH = std::min(nH, maxBounces);
    nL = std::min(nL, maxBounces);
  }
  const int hrtfLength = 2 * (nSW + nSH + nSL);
  long images = 0;
  for (int ch = 0; ch < 2; ++ch) {
    const float* d = e[ch];
    const float* v = e[2 + ch];
    const float hx = ears[0] + d[0], hy = ears[1] + d[1], hz = ears[2] + d[2];
    const float earV = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    std::vector<int64_t> acc(length, 0);
    images = room_ear(room, src, hx, hy, hz, v[0], v[1], v[2], earV, 2.0f, 2 * es, rate, length, hrtfLength,
                      filterLength, lowPass, highPass, 2 * nW, 2 * nH, 2 * nL, acc.data());
    float* out = ch == 0 ? left : right;
    for (int i = 0; i < length; ++i) out[i] = (float)acc[i] / 67108864.0f;
  }
  return images;
}

// TANMixerImpl::Mix(float**, float*) MixerImpl.cpp:226-250: out = in[0], then
// out += in[c] for c = 1.. in channel order.
void tanref_mix(const float* const* in, int channels, size_t n, float* out) {
  for (int c = 0; c < channels; ++c)
    for (size_t i = 0; i < n; ++i) out[i] = (c == 0) ? in[0][i] : out[i] + in[c][i];
}

// Mixer.cl:26-41 (device buffers): sum = 0, then sum += in[c] in channel order.
void tanref_mix_dev(const float* in, size_t stride, int channels, size_t n, float* out) {
  for (size_t i = 0; i < n; ++i) {
    float sum = 0.f;
    for (int c = 0; c < channels; ++c) sum += in[(size_t)c * stride + i];
    out[i] = sum;
  }
}

}  // extern "C"
