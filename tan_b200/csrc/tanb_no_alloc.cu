// tanb_convolve_no_alloc: one-shot multichannel FFT convolution that allocates
// no device memory.
//
// Who needs it: callers that must not allocate on the path, such as a plugin
// running inside a host application's real-time audio callback (where
// cudaMalloc can block for milliseconds and take driver locks) or a host that
// hands the library a fixed device-memory budget and forbids further
// allocation. They pass device inputs and outputs; every temporary this call
// needs (IR spectra, delay line, overlap-save history, tails, twiddles,
// descriptors) lives in the file-scope array `g_scratch` below, which every
// GPU that loads the library holds until the process exits.
//
// Limits and sharing: the whole working set of a call must fit in
// kScratchBytes (32 MiB); larger requests are refused with TANB_INVALID_ARG.
// All calls on a device share the one array and it keeps the previous call's
// contents, so this call clears what must start at zero; two calls whose work
// overlaps on the GPU (different streams, or different host threads) race on
// it -- serialise them. The first call on each device looks up the array's
// device address (once per device, with that device current); make that first
// call before any stream capture.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/tanb.h"
#include "tanb_internal.h"

namespace {

constexpr size_t kScratchBytes = TANB_NO_ALLOC_SCRATCH_BYTES;
static_assert(kScratchBytes == ((size_t)32 << 20), "the header documents a 32 MiB scratch array");
constexpr int kMaxDevices = 64;

// The scratch array. In host code `g_scratch` names a host-side stand-in, not
// device memory: host code only ever uses the address from
// cudaGetSymbolAddress (scratch_base below).
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device (looked up once per device).
cudaError_t scratch_base(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return cudaSuccess;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

// W_N^j = exp(-2 pi i j / N), computed in double with the same quadrant
// reduction as tanb::make_twiddles and rounded to float.
__global__ void twiddle_kernel(float2* tw, int N) {
  const int q4 = N / 4;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int q = j / q4, r = j % q4;
    const double th = 2.0 * 3.14159265358979323846 * (double)r / (double)N;
    double s, c;
    sincos(th, &s, &c);
    double cc, ss;
    switch (q) {
      case 0: cc = c; ss = s; break;
      case 1: cc = -s; ss = c; break;
      case 2: cc = -c; ss = -s; break;
      default: cc = s; ss = -c; break;
    }
    tw[j] = make_float2((float)cc, (float)(-ss));
  }
}

// Per-block descriptors: every channel runs with IR slot 0, no crossfade;
// rows of block b of the caller's [C][n] input and output.
__global__ void describe_kernel(tanb::ChanCtl* ctl, const float** in_rows, float** out_rows, int* chans,
                                const float* in, float* out, int C, size_t n, size_t off, int slot_new) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    ctl[c] = tanb::ChanCtl{1, 0, 0, slot_new};
    in_rows[c] = in ? in + (size_t)c * n + off : nullptr;
    out_rows[c] = out ? out + (size_t)c * n + off : nullptr;
    chans[c] = c;
  }
}

}  // namespace

extern "C" int32_t tanb_convolve_no_alloc(const float* in, const float* ir, float* out, uint32_t channels,
                                          size_t samples, size_t ir_length, uint32_t block, void* stream) {
  if (!in || !ir || !out) {
    tanb::set_last_error("tanb_convolve_no_alloc: null buffer");
    return TANB_INVALID_POINTER;
  }
  if (channels == 0 || ir_length == 0 || block < 32 || block > 8192 || (block & (block - 1)) ||
      samples % block != 0) {
    tanb::set_last_error("tanb_convolve_no_alloc: channels and ir_length must be > 0, block a power of two in "
                         "[32, 8192] and samples a multiple of block");
    return TANB_INVALID_ARG;
  }
  const size_t B = block, C = channels;
  // Reject sizes whose layout terms could wrap before forming any product:
  // every term below is at most 28 * C * P * B bytes or 24 * C * B bytes.
  const size_t P = ir_length / B + (ir_length % B != 0);
  if (C > kScratchBytes / B || P > kScratchBytes / (28 * B) || C * P > kScratchBytes / (28 * B)) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "tanb_convolve_no_alloc: %zu channels x %zu taps at block %zu exceed the scratch array of %zu bytes", C,
             ir_length, B, kScratchBytes);
    tanb::set_last_error(msg);
    return TANB_INVALID_ARG;
  }
  // scratch layout
  const size_t o_tw = 0;
  const size_t o_H = o_tw + up256(2 * B * sizeof(float2));
  const size_t o_fdl = o_H + up256(C * 2 * P * B * sizeof(float2));
  const size_t o_prev = o_fdl + up256(C * P * B * sizeof(float2));
  const size_t o_tail = o_prev + up256(C * B * sizeof(float));
  const size_t o_irp = o_tail + up256(C * 3 * B * sizeof(float2));
  const size_t o_ctl = o_irp + up256(C * P * B * sizeof(float));
  const size_t o_rows = o_ctl + up256(C * sizeof(tanb::ChanCtl));
  const size_t o_chans = o_rows + up256(2 * C * sizeof(void*));
  const size_t o_err = o_chans + up256(C * sizeof(int));
  const size_t total = o_err + 256;
  if (total > kScratchBytes) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "tanb_convolve_no_alloc: %zu channels x %zu taps at block %zu need %zu bytes of scratch; the "
             "maximum is %zu",
             C, ir_length, B, total, kScratchBytes);
    tanb::set_last_error(msg);
    return TANB_INVALID_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  cudaError_t e = scratch_base(&base);
  if (e == cudaSuccess) e = tanb::prepare_kernels();
  if (e != cudaSuccess) {
    tanb::set_last_error(cudaGetErrorString(e));
    return TANB_FAIL;
  }
  float2* tw = reinterpret_cast<float2*>(base + o_tw);
  tanb::DevState s{};
  s.B = (int)B;
  while ((1 << s.log2B) < (int)B) ++s.log2B;
  s.P = (int)P;
  s.C = (int)C;
  s.H = reinterpret_cast<float2*>(base + o_H);
  s.fdl = reinterpret_cast<float2*>(base + o_fdl);
  s.prev = reinterpret_cast<float*>(base + o_prev);
  s.tail = reinterpret_cast<float2*>(base + o_tail);
  s.tw = tw;
  s.err = reinterpret_cast<int*>(base + o_err);
  float* irp = reinterpret_cast<float*>(base + o_irp);
  tanb::ChanCtl* ctl = reinterpret_cast<tanb::ChanCtl*>(base + o_ctl);
  const float** in_rows = reinterpret_cast<const float**>(base + o_rows);
  float** out_rows = reinterpret_cast<float**>(base + o_rows + C * sizeof(void*));
  int* chans = reinterpret_cast<int*>(base + o_chans);

  // state that must start at zero (the array keeps the previous call's contents)
  do {
    if ((e = cudaMemsetAsync(s.fdl, 0, C * P * B * sizeof(float2), st)) != cudaSuccess) break;
    if ((e = cudaMemsetAsync(s.prev, 0, C * B * sizeof(float), st)) != cudaSuccess) break;
    if ((e = cudaMemsetAsync(s.tail, 0, C * 3 * B * sizeof(float2), st)) != cudaSuccess) break;
    if ((e = cudaMemsetAsync(irp, 0, C * P * B * sizeof(float), st)) != cudaSuccess) break;
    if ((e = cudaMemcpy2DAsync(irp, P * B * sizeof(float), ir, ir_length * sizeof(float),
                               ir_length * sizeof(float), C, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
      break;
    twiddle_kernel<<<(unsigned)((2 * B + 255) / 256), 256, 0, st>>>(tw, (int)(2 * B));
    // IR spectra into slot 0
    describe_kernel<<<(unsigned)((C + 127) / 128), 128, 0, st>>>(ctl, in_rows, out_rows, chans, nullptr, nullptr,
                                                                 (int)C, samples, 0, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    tanb::IrRows rows;
    rows.base = irp;
    rows.stride = (long long)(P * B);
    rows.n = (long long)(P * B);
    if ((e = tanb::launch_ir_spectrum(s, rows, chans, (int)C, ctl, st)) != cudaSuccess) break;
    int cur = 0;
    const size_t nb = samples / B;
    for (size_t b = 0; b < nb && e == cudaSuccess; ++b) {
      describe_kernel<<<(unsigned)((C + 127) / 128), 128, 0, st>>>(ctl, in_rows, out_rows, chans, in, out, (int)C,
                                                                   samples, b * B, 1);
      if ((e = cudaGetLastError()) != cudaSuccess) break;
      cur = (cur - 1 + (int)P) % (int)P;
      tanb::BlockRef ref;
      ref.ctl = ctl;
      ref.in = in_rows;
      ref.out = out_rows;
      if ((e = tanb::launch_head(s, ref, cur, (int)(b & 1), st)) != cudaSuccess) break;
      e = tanb::launch_tail(s, ref, 0, cur, (int)((b + 1) & 1), tanb::MacTiling{32, 8}, st, true);
    }
  } while (0);
  if (e != cudaSuccess) {
    tanb::set_last_error(cudaGetErrorString(e));
    return TANB_FAIL;
  }
  return TANB_OK;
}
