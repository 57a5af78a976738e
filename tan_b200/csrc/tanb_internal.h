// Internal interface between the host engine (tanb_convolution.cpp) and the
// sm_100a kernels (tanb_kernels.cu). Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <mutex>

// A TAN context: the CUDA device its objects run on.
struct tanb_context {
  int device = 0;
};

namespace tanb {

// Records the text returned by tanb_last_error() on this thread.
void set_last_error(const char* msg);

// An NVTX range over a scope: the entry points name their host work so that
// Nsight tools (and ncu's --nvtx filters) can place it; without a tool
// attached a push or pop costs a few nanoseconds.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// A set-up step that must run once on every CUDA device a process uses (kernel
// attributes such as the dynamic shared-memory limit are held per device):
// run(f) calls f() the first time it is called with a given device current
// and returns that result on every later call on the same device.
class OncePerDevice {
 public:
  template <class F>
  cudaError_t run(F&& f) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu_);
    if (!done_[dev]) {
      res_[dev] = f();
      done_[dev] = true;
    }
    return res_[dev];
  }

 private:
  static constexpr int kMaxDevices = 64;
  std::mutex mu_;
  bool done_[kMaxDevices] = {};
  cudaError_t res_[kMaxDevices] = {};
};

// Per-channel control word for one audio block, uploaded with the block's input.
//   run       channel is processed this block (reference: !m_availableChannels[c])
//   swap      a new IR takes effect this block (crossfade from slot_cur to slot_new)
//   slot_cur  IR slot in use before this block
//   slot_new  IR slot holding the pending IR
struct ChanCtl {
  int32_t run;
  int32_t swap;
  int32_t slot_cur;
  int32_t slot_new;
};

// Error codes a kernel writes to DevState::err.
enum : int { kErrNone = 0, kErrBulkWaitTimeout = 1 };

// Polls of an mbarrier before a bounded wait gives up (about a second).
constexpr int kBulkWaitLimit = 1 << 20;

// Device-resident state of one convolution object.
// Spectra are "packed" half spectra of a 2B-point real FFT: B complex bins,
// bin 0 holding (X[0].re, X[B].re) -- both are real.
struct DevState {
  int B;          // block size (power of two)
  int log2B;
  int P;          // partitions = ceil(L / B), at least 1
  int C;          // channels
  float2* H;      // IR spectra      [C][2 slots][P][B]
  float2* fdl;    // delay line      [C][P][B]  (slot (cur + i) mod P holds X_{k-i})
  float* prev;    // previous input  [C][B]     (overlap-save history)
  float2* tail;   // tails           [C][2][B]  ([0]: active IR, [1]: pending IR)
  const float2* tw;  // W_N^j, N = 2B, j in [0, N)
  int* err;       // device-visible error word (host-mapped); nonzero after a
                  // bounded wait in a kernel gave up (kErr* codes)
  int wait_limit = kBulkWaitLimit;  // polls of a bounded wait for a pipeline
                                    // stage before it gives up (a test hook
                                    // lowers it; draining in-flight copies
                                    // always uses kBulkWaitLimit)
};



__host__ __device__ inline size_t h_index(const DevState& s, int c, int slot, int part) {
  return (((size_t)c * 2 + slot) * s.P + part) * s.B;
}

// Tiling of the tail multiply-accumulate: UX units (float4 = 2 bins) by SY
// partition splits per CTA (UX * SY threads), each thread keeping `depth`
// partitions' loads in flight.
struct MacTiling {
  int ux;         // kind 0: float4 units per CTA row; kind 1: bins per CTA / 2
  int sy;         // kind 0: partition splits per CTA; kind 1: pipeline stages
  int depth = 4;  // kind 0: partitions in flight per thread; kind 1: rows per stage
  int kind = 0;   // 0: register loads (LDG.128); 1: cp.async.bulk into shared memory
};

// Tilings the tail kernel is compiled for (index -> MacTiling).
int mac_tiling_count();
MacTiling mac_tiling(int index);

// Per-block descriptors of up to kParamChannels channels, passed to the head
// and tail kernels as a kernel parameter (no copy to device memory and no
// dependent global load before a CTA knows its channel's state). The launch
// cost grows with the parameter size (two launches with 4 KiB of parameters
// took 11.9 us to enqueue against 4.8 us with 256 B), so a channel's state is
// one byte, the tail gets only those bytes, and host rows in the object's
// staging are described by two base pointers instead of pointer tables.
constexpr int kParamChannels = 128;
enum : uint8_t { kCtlRun = 1, kCtlSwap = 2, kCtlSlotCur = 4, kCtlSlotNew = 8, kCtlHasIn = 16 };
inline uint8_t pack_ctl(const ChanCtl& c, bool has_in) {
  return (uint8_t)((c.run ? kCtlRun : 0) | (c.swap ? kCtlSwap : 0) | (c.slot_cur ? kCtlSlotCur : 0) |
                   (c.slot_new ? kCtlSlotNew : 0) | (has_in ? kCtlHasIn : 0));
}
struct CtlParam {
  uint8_t ctl[kParamChannels];
};
// Caller rows: per-channel pointers.
struct ParamDesc {
  CtlParam c;
  const float* in[kParamChannels];
  float* out[kParamChannels];
};
// Rows at fixed strides (the object's staging, or the caller's rows when they
// sit in one pinned host allocation): channel c reads in + c * stride (when
// kCtlHasIn is set) and writes out + c * ostride.
struct StageDesc {
  CtlParam c;
  const float* in;
  float* out;
  long long stride;
  long long ostride;
};

// Where a launch finds its per-channel descriptors: a ParamDesc or StageDesc
// (host copy, passed by value), a CtlParam (tail launches that need only the
// channel states), or device arrays.
struct BlockRef {
  const ParamDesc* param = nullptr;
  const StageDesc* stage = nullptr;
  const CtlParam* ctlp = nullptr;
  const ChanCtl* ctl = nullptr;
  const float* const* in = nullptr;
  float* const* out = nullptr;
  // the channel states of a parameter descriptor, whichever kind it is
  const CtlParam* ctl_param() const { return param ? &param->c : stage ? &stage->c : ctlp; }
};

// Fused PCM pipeline in the head kernel (tanb_convolution_process_mix_pcm16).
// Inputs are int16 rows converted with in_scale (the host short->float
// converter's rule); each channel's output row (the descriptor's out: device
// scratch) is mixed into its group by the last head CTA of that group to finish
// (sum from 0 in ascending channel order, the device mixer's rule) and converted
// to int16 with out_scale (the device float->short rule) into out16 + g * B.
struct MixEpi {
  int active = 0;
  float in_scale = 0.f;            // gain / 32767
  float out_scale = 0.f;           // 32767 * gain
  const int* chan_group = nullptr; // [C]
  const int* gstart = nullptr;     // [ngroups + 1] into gchan
  const int* gchan = nullptr;      // [C] channels of each group, ascending
  unsigned* count = nullptr;       // [ngroups] head CTAs of the group done this block
  const float* scratch = nullptr;  // [C][B] channel outputs
  int16_t* out16 = nullptr;        // [ngroups][B]
  int* clip = nullptr;             // set when a sample was clamped
};

// Completion signal of a head launch for host-row calls: every CTA fences its
// output stores system-wide and counts itself in `count` (device memory, zero
// between launches); the last one resets the count and stores `seq` into
// `flag` (mapped host memory). The host then reads the outputs without waiting
// for the tail launched behind the head. seq == 0: no signal.
struct HeadSignal {
  unsigned* count = nullptr;
  long long* flag = nullptr;
  long long seq = 0;
};

// Where the IR-spectrum kernel reads row j (the IR of channel chans[j]):
// ptrs[j] when ptrs (a device array) is set, else base + j * stride. Samples
// at and after n read as zero, so rows need no padding to P*B.
struct IrRows {
  const float* base = nullptr;
  long long stride = 0;
  const float* const* ptrs = nullptr;
  long long n = 0;
};

// R2C of each IR partition into slot `slot_new` of the channels listed in
// `chans` (device array of nch channel indices).
cudaError_t launch_ir_spectrum(const DevState& s, const IrRows& ir, const int* chans, int nch,
                               const ChanCtl* ctl, cudaStream_t st);

// Head of one block for every running channel: FFT of [prev, x], insert into
// delay-line slot `cur`, multiply with partitions 0 and 1 (X_k, X_{k-1}), add
// the block's tail (row `parity` = block index & 1, and row 2 for a pending IR
// on swap channels), inverse FFT, overlap-save output (and the crossfade).
// `in[c]` / `out[c]` are device pointers to channel c's B input / output samples.
cudaError_t launch_head(const DevState& s, const BlockRef& d, int cur, int parity, cudaStream_t st,
                        const MixEpi& epi = MixEpi{}, const HeadSignal& sig = HeadSignal{});

// Tail multiply-accumulate, partitions 2..P-1, for the block after the one
// whose spectrum sits in delay-line slot `cur`:
//   tail[c][trow] = sum_{i=2}^{P-1} FDL[c][(cur + i - 1) mod P] * H[c][slot][i]
// which = 0: running channels, slot = swap ? slot_new : slot_cur, trow = the
//            next block's parity
// which = 1: channels with swap set (pending IR), slot = slot_new, trow = 2;
//            `cur` is then the newest slot before the coming block
// It reads only X_{k-1} and older and writes a row the head of block k does not
// read, so it shares no data with that head. pdl: launch with programmatic
// stream serialization, directly behind the head of the same block (the two
// then run side by side); every other launch passes false.
cudaError_t launch_tail(const DevState& s, const BlockRef& d, int which, int cur, int trow, MacTiling t,
                        cudaStream_t st, bool pdl = false);

// Per-channel descriptor of one TIME_DOMAIN call.
struct TdChan {
  const float* in;      // device row of n input samples (null: silence)
  float* out;           // device row of n outputs (null: discarded)
  const float* ir;      // device IR row, taps [first, last) valid
  const float* ir_new;  // second IR on a crossfade call
  int32_t pos;          // history position before this call
  int32_t first, last;  // tap range
  int32_t run;          // channel processed
  int32_t swap;         // crossfade ir -> ir_new
  int32_t fade0;        // crossfade sample index of this call's first output
  int32_t pad[2];
};

// TIME_DOMAIN: append n input samples to each running channel's circular
// history (len samples, [C][len]) and compute n direct-FIR outputs.
cudaError_t launch_td(float* hist, int len, const TdChan* ch, int C, int n, int fade_len, cudaStream_t st);

// Sets the shared-memory attributes of every kernel (once per device).
cudaError_t prepare_kernels();

// Fills the twiddle table W_N^j = exp(-2 pi i j / N) on the host, computed in
// double and rounded to float, exact at multiples of pi/2.
void make_twiddles(int N, float2* out);

}  // namespace tanb
