// Host engine behind include/tanb.h: the TANConvolution state machine of the
// reference (tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp)
// driving the sm_100a kernels of tanb_kernels.cu on one CUDA stream per object.
//
// Per Process call the host
//   1. runs the channel-flag bookkeeping per block (ConvolutionImpl.cpp:2867-2907),
//   2. writes one descriptor per block (per-channel run / swap / IR slots and
//      the input and output row pointers): a kernel parameter for up to 128
//      channels, else pinned staging copied to the device in one transfer,
//   3. for host rows, copies the inputs into pinned staging that the head
//      kernel reads in place and points the outputs at pinned staging that it
//      writes in place (no separate host<->device copies),
//   4. enqueues per block the head and, behind it, the tail (programmatic
//      dependent launch, so the two overlap), and waits for the last of them.
// UpdateResponseTD transforms the new IR into the idle slot and precomputes
// that IR's tail, so the swap block costs the same device time as any other.
#include <cuda.h>  // CUpointer_attribute values only; the driver call is resolved at run time
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include "../../include/tanb.h"
#include "tanb_engine_host.h"
#include "tanb_host_pool.h"
#include "tanb_internal.h"

using tanb::ChanCtl;
using tanb::DevState;
using tanb::MacTiling;

namespace {

thread_local std::string g_last_error;

}  // namespace

// Every reported failure also clears the CUDA runtime's per-thread last error:
// a failed runtime call leaves it set, and the next launch check
// (cudaGetLastError after a launch) would otherwise report that stale error.
void tanb::set_last_error(const char* msg) {
  g_last_error = msg;
  cudaGetLastError();
}

namespace {

int32_t fail(int32_t code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  tanb::set_last_error(buf);
  return code;
}

#define TANB_CUDA(expr)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(e_ == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL,       \
                  "%s failed: %s", #expr, cudaGetErrorString(e_));                       \
  } while (0)

constexpr int kMaxBlocksPerChunk = 8;
// Host-row IR updates of at least this many bytes are staged on the host pool
// in kStageGroups channel groups.
constexpr size_t kParallelStageBytes = 1u << 20;
constexpr int kStageGroups = 4;
constexpr uint32_t kStopInput = TANB_CHANNEL_FLAG_STOP_INPUT;
constexpr uint32_t kFlush = TANB_CHANNEL_FLAG_FLUSH_STREAM;

enum class Mem { Host, Device };

}  // namespace

struct tanb_convolution {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  // host microseconds of the last uniform Process call by part, and which of
  // its caller rows the kernels addressed in place (tanb_convolution_call_times)
  double ct[6] = {0, 0, 0, 0, 0, 0};
  bool initialized = false;
  bool terminated = false;
  bool finalize_mode = false;
  bool finalize_due = false;
  uint32_t method = 0;
  int L = 0, B = 0, C = 0, P = 0, length = 0;
  cudaStream_t stream = nullptr;
  DevState ds{};
  float2* d_tw = nullptr;
  MacTiling tiling{32, 8};
  size_t dev_bytes = 0;

  // host mirror of the per-channel state
  std::vector<int> active, pending, slot_new, tail_left;
  std::vector<uint8_t> available, flushed;
  int cur = 0;  // delay-line slot of the newest spectrum

  // Process staging: pinned [kMaxBlocksPerChunk] descriptors, then inputs;
  // pinned outputs; the device copy of the descriptors (more than 128 channels)
  size_t desc_bytes = 0;
  uint8_t* h_stage = nullptr;
  uint8_t* d_stage = nullptr;
  float* h_out = nullptr;
  const ChanCtl* last_desc = nullptr;  // device descriptor of the last head (for ProcessFinalize)
  int last_cur = 0;
  int64_t blocks = 0;  // blocks processed: the parity selects the tail row
  // per-block descriptors passed as kernel parameters (C <= kParamChannels)
  std::vector<tanb::ParamDesc> pdesc;
  std::vector<tanb::StageDesc> sdesc;
  // Process's per-call bookkeeping, sized at Init so that a call allocates
  // nothing: running / flushed channels of the current block and of each
  // block of a chunk, and each block's delay-line slot
  std::vector<uint8_t> scr_run, scr_flush;
  std::vector<std::vector<uint8_t>> scr_run_b;
  std::vector<std::vector<int>> scr_flush_b;
  std::vector<int> scr_cur_b;
  tanb::CtlParam last_ctlp{};
  bool last_is_param = false;

  // UpdateResponseTD staging: IR rows [C][P*B], then ChanCtl[C] + int[C]
  float* h_ir = nullptr;
  float* d_ir = nullptr;
  int* h_err = nullptr;  // host-mapped error word written by kernels (DevState::err)
  // head completion for host-row calls (tanb::HeadSignal): the count lives in
  // device memory, the flag in mapped host memory; head_seq numbers launches
  unsigned* d_head_count = nullptr;
  long long* h_head_flag = nullptr;
  long long* d_head_flag = nullptr;
  long long head_seq = 0;
  // host staging rows may still be in use by heads whose completion this
  // object has not observed (ev_out covers them)
  bool staging_busy = false;
  uint8_t* h_uctl = nullptr;
  uint8_t* d_uctl = nullptr;

  cudaEvent_t ev_stage = nullptr, ev_ir = nullptr, ev_out = nullptr;

  // fused PCM pipeline (tanb_convolution_process_mix_pcm16), allocated on first use
  float* d_mix_scratch = nullptr;   // [C][B] channel outputs
  int* d_mix_table = nullptr;       // chan_group[C], gstart[C + 1], gchan[C], count[C]
  int* h_clip = nullptr;            // host-mapped clip flag
  std::vector<uint32_t> mix_groups; // group map the table holds

  // Non-uniform methods: a private batched engine holding one non-uniformly
  // partitioned session of C channels (slots [0, C)); the channel-flag
  // bookkeeping stays here. Row tables for device rows: pinned [8 blocks][2][C]
  // (inputs, outputs) and their device copy.
  tanb_engine* nu_eng = nullptr;
  int32_t nu_sess = -1;
  float* nu_in = nullptr;    // the engine's pinned input rows [C][B]
  float* nu_out = nullptr;   // the engine's pinned output rows [C][B]
  const float** h_nu_tab = nullptr;
  const float** d_nu_tab = nullptr;
  std::vector<uint32_t> nu_blocks, nu_parts;

  // TIME_DOMAIN method state (history of `length` samples per channel)
  bool td = false;
  float* td_hist = nullptr;    // [C][length]
  float* td_ir = nullptr;      // [2 slots][C][length]  (Process IRs)
  float* td_dir = nullptr;     // [C][length]           (ProcessDirect per-call IRs)
  float* td_io = nullptr;      // [2][C][length]        (device in / out staging)
  float* h_td = nullptr;       // pinned [3][C][length] (IR, in, out staging)
  tanb::TdChan* d_tdchan = nullptr;
  tanb::TdChan* h_tdchan = nullptr;
  std::vector<int> td_pos;
  int td_fade = -1;            // crossfade sample index, -1 when none
  std::vector<int> td_swapping;

  // kernel accounting: launch counts always, device time when profiling is on
  enum Kind { kHead = 0, kTail = 1, kIr = 2, kKinds = 3 };
  int64_t launches[kKinds] = {0, 0, 0};
  bool profiling = false;
  struct Timed {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Timed> timed;          // recorded, not yet read
  std::vector<cudaEvent_t> ev_pool;  // free events
  double ms[kKinds] = {0, 0, 0};
  int64_t timed_count[kKinds] = {0, 0, 0};

  // descriptor accessors
  ChanCtl* desc_ctl(uint8_t* base, int b) { return reinterpret_cast<ChanCtl*>(base + b * desc_bytes); }
  const float** desc_in(uint8_t* base, int b) {
    return reinterpret_cast<const float**>(base + b * desc_bytes + sizeof(ChanCtl) * C);
  }
  float** desc_out(uint8_t* base, int b) {
    return reinterpret_cast<float**>(base + b * desc_bytes + (sizeof(ChanCtl) + sizeof(void*)) * C);
  }
  float* stage_in(uint8_t* base, int b, int c) {
    return reinterpret_cast<float*>(base + kMaxBlocksPerChunk * desc_bytes) + ((size_t)b * C + c) * B;
  }
};

namespace {

cudaEvent_t pool_event(tanb_convolution* v) {
  if (!v->ev_pool.empty()) {
    cudaEvent_t e = v->ev_pool.back();
    v->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Runs `launch` on the object's stream, counting it and, when profiling, timing
// it with an event pair on the same stream.
template <typename F>
cudaError_t counted(tanb_convolution* v, int kind, F&& launch) {
  v->launches[kind] += 1;
  if (!v->profiling) return launch();
  cudaEvent_t a = pool_event(v), b = pool_event(v);
  cudaEventRecord(a, v->stream);
  cudaError_t e = launch();
  cudaEventRecord(b, v->stream);
  v->timed.push_back({kind, a, b});
  return e;
}

void drain_timed(tanb_convolution* v) {
  for (auto& t : v->timed) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      v->ms[t.kind] += ms;
      v->timed_count[t.kind] += 1;
    }
    v->ev_pool.push_back(t.a);
    v->ev_pool.push_back(t.b);
  }
  v->timed.clear();
}

void free_all(tanb_convolution* v) {
  if (v->nu_eng) tanb_engine_release(v->nu_eng);
  v->nu_eng = nullptr;
  v->nu_sess = -1;
  v->nu_in = v->nu_out = nullptr;
  cudaFreeHost(v->h_nu_tab);
  cudaFree(v->d_nu_tab);
  v->h_nu_tab = v->d_nu_tab = nullptr;
  if (v->stream) cudaStreamSynchronize(v->stream);
  drain_timed(v);
  for (cudaEvent_t e : v->ev_pool) cudaEventDestroy(e);
  v->ev_pool.clear();
  cudaFree(v->ds.H);
  cudaFree(v->ds.fdl);
  cudaFree(v->ds.prev);
  cudaFree(v->ds.tail);
  cudaFree(v->d_tw);
  cudaFree(v->d_stage);
  cudaFree(v->d_head_count);
  v->d_head_count = nullptr;
  cudaFree(v->d_ir);
  cudaFree(v->d_uctl);
  cudaFree(v->d_mix_scratch);
  cudaFree(v->d_mix_table);
  cudaFreeHost(v->h_clip);
  v->d_mix_scratch = nullptr;
  v->d_mix_table = nullptr;
  v->h_clip = nullptr;
  v->mix_groups.clear();
  cudaFreeHost(v->h_stage);
  cudaFreeHost(v->h_out);
  cudaFreeHost(v->h_ir);
  cudaFreeHost(v->h_uctl);
  cudaFreeHost(v->h_err);
  v->h_err = nullptr;
  cudaFreeHost(v->h_head_flag);
  v->h_head_flag = v->d_head_flag = nullptr;
  v->staging_busy = false;
  cudaFree(v->td_hist);
  cudaFree(v->td_ir);
  cudaFree(v->td_dir);
  cudaFree(v->td_io);
  cudaFree(v->d_tdchan);
  cudaFreeHost(v->h_td);
  cudaFreeHost(v->h_tdchan);
  v->td_hist = v->td_ir = v->td_dir = v->td_io = v->h_td = nullptr;
  v->d_tdchan = v->h_tdchan = nullptr;
  if (v->ev_stage) cudaEventDestroy(v->ev_stage);
  if (v->ev_ir) cudaEventDestroy(v->ev_ir);
  if (v->ev_out) cudaEventDestroy(v->ev_out);
  if (v->stream) cudaStreamDestroy(v->stream);
  v->ds = DevState{};
  v->d_tw = nullptr;
  v->d_stage = v->h_stage = nullptr;
  v->h_out = nullptr;
  v->d_ir = v->h_ir = nullptr;
  v->d_uctl = v->h_uctl = nullptr;
  v->ev_stage = v->ev_ir = v->ev_out = nullptr;
  v->stream = nullptr;
  v->last_desc = nullptr;
  v->dev_bytes = 0;
}

template <typename T>
cudaError_t dev_alloc(tanb_convolution* v, T** p, size_t count) {
  size_t bytes = count * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
  if (e == cudaSuccess) {
    v->dev_bytes += bytes;
    e = cudaMemsetAsync(*p, 0, bytes, v->stream);
  }
  return e;
}

MacTiling default_tiling(int B, int P) {
  const int U = B / 2;
  if (P >= 256 && U >= 32) return {32, 16, 4};
  if (U >= 32) return {32, 8, 4};
  return {16, 16, 4};
}

// Zeroes one channel's delay line, history and tails (intended flush semantics;
// the reference's CPU flush is ConvolutionImpl.cpp:1261-1351).
cudaError_t flush_channel(tanb_convolution* v, int c) {
  cudaError_t e;
  const size_t B = v->B, P = v->P;
  if ((e = cudaMemsetAsync(v->ds.fdl + (size_t)c * P * B, 0, P * B * sizeof(float2), v->stream)) != cudaSuccess)
    return e;
  if ((e = cudaMemsetAsync(v->ds.prev + (size_t)c * B, 0, B * sizeof(float), v->stream)) != cudaSuccess) return e;
  return cudaMemsetAsync(v->ds.tail + (size_t)c * 3 * B, 0, 3 * B * sizeof(float2), v->stream);
}

int32_t run_pending_finalize(tanb_convolution* v) {
  if (!v->finalize_due) return TANB_OK;
  v->finalize_due = false;
  if (v->P <= 2) return TANB_OK;  // no partitions beyond the head's two
  tanb::BlockRef ref;
  if (v->last_is_param)
    ref.ctlp = &v->last_ctlp;
  else
    ref.ctl = v->last_desc;
  TANB_CUDA(counted(v, tanb_convolution::kTail,
                    [&] {
                      return tanb::launch_tail(v->ds, ref, 0, v->last_cur, (int)(v->blocks & 1), v->tiling,
                                               v->stream);
                    }));
  return TANB_OK;
}

int32_t td_update(tanb_convolution* v, Mem mem, const float* const* ir, size_t n, const uint32_t* flags,
                  uint32_t op);
int32_t td_process(tanb_convolution* v, Mem in_mem, const float* const* in, Mem out_mem, float* const* out,
                   size_t n, const uint32_t* flags, size_t* done);
int channel_flags(tanb_convolution* v, const uint32_t* flags, std::vector<uint8_t>& run,
                  std::vector<uint8_t>& flush);
int32_t nu_update(tanb_convolution* v, Mem mem, const float* const* ir, size_t n, const uint32_t* flags);
int32_t nu_process(tanb_convolution* v, Mem in_mem, const float* const* in, Mem out_mem, float* const* out,
                   size_t n, const uint32_t* flags, size_t* done);

// ---------------------------------------------------------------------------
// Caller rows in page-locked host memory. When every row of a call sits at one
// stride inside one pinned allocation that the device addresses at the same
// virtual addresses, the head reads (and writes) the rows in place over the
// bus instead of through the object's staging: no host copy in, none out.
// Anything else -- pageable rows, rows spread over several allocations,
// unequal strides, misalignment, input and output spans that overlap -- takes
// the staging path.
// ---------------------------------------------------------------------------
using PtrAttrsFn = CUresult (*)(unsigned int, CUpointer_attribute*, void**, CUdeviceptr);

PtrAttrsFn ptr_attrs_fn() {
  static const PtrAttrsFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuPointerGetAttributes", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      (void)cudaGetLastError();
      return static_cast<PtrAttrsFn>(nullptr);
    }
    return reinterpret_cast<PtrAttrsFn>(f);
  }();
  return fn;
}

// True when the bytes [lo, hi) lie in one page-locked host allocation that the
// device addresses at the same virtual addresses: one driver query of the
// first byte (memory type, managed or not, its device address, the range of
// its allocation). An address the driver does not know (pageable memory)
// comes back with the default values, which fail the test. Within one
// allocation the device mapping is one linear range, so identity at `lo`
// holds for every byte up to `hi`.
bool pinned_span(const void* lo, const void* hi) {
  const PtrAttrsFn fn = ptr_attrs_fn();
  if (!fn || hi <= lo) return false;
  unsigned int mem_type = 0, managed = 0;
  CUdeviceptr dptr = 0, start = 0;
  size_t size = 0;
  CUpointer_attribute attrs[5] = {CU_POINTER_ATTRIBUTE_MEMORY_TYPE, CU_POINTER_ATTRIBUTE_IS_MANAGED,
                                  CU_POINTER_ATTRIBUTE_DEVICE_POINTER, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR,
                                  CU_POINTER_ATTRIBUTE_RANGE_SIZE};
  void* data[5] = {&mem_type, &managed, &dptr, &start, &size};
  const CUdeviceptr l = (CUdeviceptr) reinterpret_cast<uintptr_t>(lo);
  const CUdeviceptr h = (CUdeviceptr) reinterpret_cast<uintptr_t>(hi);
  if (fn(5, attrs, data, l) != CUDA_SUCCESS) return false;
  return mem_type == CU_MEMORYTYPE_HOST && !managed && dptr == l && l >= start && h <= start + size;
}

struct PinnedRows {
  const float* base = nullptr;  // row c is base + c * stride (listed rows only)
  long long stride = 0;
  uintptr_t lo = 0, hi = 0;     // bytes the call reads or writes
};

// Rows of n samples each at one stride in one pinned, identity-mapped host
// allocation; null rows allowed when `nulls`.
bool pinned_rows(const float* const* rows, int C, size_t n, bool nulls, PinnedRows* out) {
  int c0 = -1, c1 = -1;
  for (int c = 0; c < C; ++c) {
    if (rows[c]) {
      if (c0 < 0) c0 = c;
      c1 = c;
    } else if (!nulls) {
      return false;
    }
  }
  if (c0 < 0 || n == 0) return false;
  // byte offsets, so that a row off the float grid is seen as such
  auto at = [&](int c) { return (long long)reinterpret_cast<uintptr_t>(rows[c]); };
  long long s = 0;  // stride in floats
  if (c1 > c0) {
    const long long d = at(c1) - at(c0);
    if (d <= 0 || d % (4LL * (c1 - c0))) return false;
    s = d / (4LL * (c1 - c0));
    if (s < (long long)n) return false;  // overlapping rows
    for (int c = c0 + 1; c < c1; ++c)
      if (rows[c] && at(c) - at(c0) != 4 * s * (c - c0)) return false;
  }
  if ((at(c0) & 15) || ((s * 4) & 15)) return false;
  if (!pinned_span(rows[c0], rows[c1] + n)) return false;
  out->stride = s;
  // row c is base + c * stride for the listed rows; the base itself is only an
  // address the kernels offset from (it may precede the first listed row)
  out->base = reinterpret_cast<const float*>(reinterpret_cast<uintptr_t>(rows[c0]) -
                                             (uintptr_t)(4LL * c0 * s));
  out->lo = reinterpret_cast<uintptr_t>(rows[c0]);
  out->hi = reinterpret_cast<uintptr_t>(rows[c1] + n);
  return true;
}

// Per-update descriptors, one upload: [ChanCtl x C][int channel list x C]
// [8-byte aligned: IR row pointers x C].
size_t uctl_ptr_offset(size_t C) { return ((sizeof(ChanCtl) + sizeof(int)) * C + 7) & ~size_t(7); }
size_t uctl_bytes(size_t C) { return uctl_ptr_offset(C) + C * sizeof(void*); }

int32_t update_common(tanb_convolution* v, Mem mem, const float* const* ir, size_t n, const uint32_t* flags,
                      uint32_t op) {
  tanb::NvtxRange range("tanb UpdateResponseTD");
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "UpdateResponseTD before Init");
  if (!ir) return fail(TANB_INVALID_ARG, "ppBuffer == NULL");
  if (n > (size_t)v->L) return fail(TANB_INVALID_ARG, "IR length %zu exceeds Init length %d", n, v->L);
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  if (v->td) return td_update(v, mem, ir, n, flags, op);
  if (v->nu_eng) return nu_update(v, mem, ir, n, flags);
  if (run_pending_finalize(v) != TANB_OK) return TANB_FAIL;

  const int C = v->C;
  std::vector<int> chans;
  for (int c = 0; c < C; ++c) {
    if (flags && (flags[c] & kFlush)) TANB_CUDA(flush_channel(v, c));
    if (flags && (flags[c] & kStopInput)) continue;
    if (!ir[c] && n > 0) return fail(TANB_INVALID_ARG, "ppBuffer[%d] == NULL", c);
    chans.push_back(c);
  }
  if (chans.empty()) return TANB_OK;

  TANB_CUDA(cudaEventSynchronize(v->ev_ir));
  const int nch = (int)chans.size();
  tanb::IrRows rows;
  rows.n = (long long)n;
  PinnedRows pin;
  const bool direct = mem == Mem::Host && n && nch == C && pinned_rows(ir, C, n, false, &pin);
  if (direct) {
    // rows in one pinned allocation at one stride: a single strided transfer
    // into the compact rows, no host copy (the call waits for the transfer,
    // so that the caller's rows are free again when it returns)
    TANB_CUDA(cudaMemcpy2DAsync(v->d_ir, n * sizeof(float), pin.base, (size_t)pin.stride * sizeof(float),
                                n * sizeof(float), (size_t)C, cudaMemcpyHostToDevice, v->stream));
    rows.base = v->d_ir;
    rows.stride = (long long)n;
  } else if (mem == Mem::Host) {
    // Compact staging (row stride n; the kernel reads zeros past n). Large
    // updates copy rows on the host pool in channel groups and send each group
    // as soon as it is staged, so its transfer overlaps the next group's copy.
    const size_t row_bytes = n * sizeof(float);
    const int groups = (row_bytes * nch >= kParallelStageBytes) ? std::min(nch, kStageGroups) : 1;
    for (int q = 0; q < groups && n; ++q) {
      const int j0 = (int)((long long)nch * q / groups), j1 = (int)((long long)nch * (q + 1) / groups);
      if (groups > 1) {
        tanb::host_parallel_for(j1 - j0, [&](int r) {
          tanb::copy_for_device(v->h_ir + (size_t)(j0 + r) * n, ir[chans[j0 + r]], row_bytes);
        });
      } else {
        for (int j = j0; j < j1; ++j) tanb::copy_for_device(v->h_ir + (size_t)j * n, ir[chans[j]], row_bytes);
      }
      TANB_CUDA(cudaMemcpyAsync(v->d_ir + (size_t)j0 * n, v->h_ir + (size_t)j0 * n, (size_t)(j1 - j0) * row_bytes,
                                cudaMemcpyHostToDevice, v->stream));
    }
    rows.base = v->d_ir;
    rows.stride = (long long)n;
  } else {
    // the kernel reads the caller's rows in place
    const float** up = reinterpret_cast<const float**>(v->h_uctl + uctl_ptr_offset(C));
    for (int j = 0; j < nch; ++j) up[j] = ir[chans[j]];
    rows.ptrs = reinterpret_cast<const float* const*>(v->d_uctl + uctl_ptr_offset(C));
  }
  for (int c : chans) {
    if (!v->pending[c]) {
      v->slot_new[c] = 1 - v->active[c];
      v->pending[c] = 1;
    }
  }
  ChanCtl* uctl = reinterpret_cast<ChanCtl*>(v->h_uctl);
  int* uch = reinterpret_cast<int*>(v->h_uctl + sizeof(ChanCtl) * C);
  for (int c = 0; c < C; ++c) uctl[c] = ChanCtl{v->pending[c], v->pending[c], v->active[c], v->slot_new[c]};
  for (int j = 0; j < nch; ++j) uch[j] = chans[j];
  TANB_CUDA(cudaMemcpyAsync(v->d_uctl, v->h_uctl, uctl_bytes(C), cudaMemcpyHostToDevice, v->stream));
  TANB_CUDA(cudaEventRecord(v->ev_ir, v->stream));
  const ChanCtl* d_uctl = reinterpret_cast<const ChanCtl*>(v->d_uctl);
  const int* d_uch = reinterpret_cast<const int*>(v->d_uctl + sizeof(ChanCtl) * C);
  TANB_CUDA(counted(v, tanb_convolution::kIr,
                    [&] { return tanb::launch_ir_spectrum(v->ds, rows, d_uch, nch, d_uctl, v->stream); }));
  // tail of the pending IR for the next block, from the current delay line
  if (v->P > 2)
    TANB_CUDA(counted(v, tanb_convolution::kTail,
                      [&] {
                        tanb::BlockRef ref;
                        ref.ctl = d_uctl;
                        return tanb::launch_tail(v->ds, ref, 1, v->cur, 2, v->tiling, v->stream);
                      }));
  if (op & TANB_OPERATION_FLAG_BLOCK_UNTIL_READY)
    TANB_CUDA(cudaStreamSynchronize(v->stream));
  else if (direct)
    TANB_CUDA(cudaEventSynchronize(v->ev_ir));  // behind the transfer from the caller's rows
  return TANB_OK;
}

// Per-block channel-flag bookkeeping, ConvolutionImpl.cpp:2867-2907 with
// per-channel state. Returns the number of running channels; fills run[] and
// flush[] (channels whose state is cleared before this block).
int channel_flags(tanb_convolution* v, const uint32_t* flags, std::vector<uint8_t>& run,
                  std::vector<uint8_t>& flush) {
  int nrun = 0;
  for (int c = 0; c < v->C; ++c) {
    flush[c] = 0;
    const uint32_t f = flags ? flags[c] : 0u;
    const bool was_free = v->available[c] != 0;
    if (!flags) {
      v->available[c] = 0;
      v->tail_left[c] = v->length;
    } else if (f & kStopInput) {
      if (f & kFlush) {
        v->available[c] = 1;
        v->tail_left[c] = 0;
      } else if (v->tail_left[c] > 0) {
        v->available[c] = 0;
        v->tail_left[c] -= v->B;
        if (v->tail_left[c] <= 0) flush[c] = 1;
      } else {
        v->available[c] = 1;
        v->tail_left[c] = 0;
      }
    } else {
      v->available[c] = 0;
      v->tail_left[c] = v->length;
    }
    if (flags && (f & kFlush)) {
      if (!v->flushed[c]) flush[c] = 1;
      v->flushed[c] = 1;
    } else {
      v->flushed[c] = 0;
    }
    run[c] = !v->available[c];
    // a free channel that starts running again starts from silence
    if (was_free && run[c]) flush[c] = 1;
    nrun += run[c];
  }
  return nrun;
}

// Waits until the head launch numbered `seq` has signalled (tanb::HeadSignal).
// Spins on the mapped flag; every 256 polls it also asks whether ev_out (behind
// the tail launched after that head) has completed, so a failed launch or a
// missing signal ends the wait with an error instead of spinning on.
int32_t wait_heads(tanb_convolution* v, long long seq) {
  volatile long long* flag = v->h_head_flag;
  for (unsigned n = 1;; ++n) {
    if (*flag >= seq) {
      std::atomic_thread_fence(std::memory_order_acquire);
      return TANB_OK;
    }
    if ((n & 255) == 0) {
      const cudaError_t e = cudaEventQuery(v->ev_out);
      if (e == cudaSuccess) {
        if (*flag >= seq) continue;
        return fail(TANB_FAIL, "head launch %lld completed without signalling", seq);
      }
      if (e != cudaErrorNotReady) return fail(TANB_FAIL, "head wait: %s", cudaGetErrorString(e));
    }
#if defined(__x86_64__)
    _mm_pause();
#endif
  }
}

// Rows and rules of the fused PCM pipeline (tanb_convolution_process_mix_pcm16).
struct PcmIO {
  const int16_t* const* in;
  size_t in_step;
  float in_gain;
  const uint32_t* group;
  uint32_t ngroups;
  int16_t* const* out;
  size_t out_step;
  float out_gain;
};

// Device table of the group map (channels of each group in ascending order)
// and the fused pipeline's scratch; uploaded when the map changes.
cudaError_t ensure_mix(tanb_convolution* v, const PcmIO& pcm, tanb::MixEpi* epi) {
  const int C = v->C, B = v->B;
  cudaError_t e;
  if (!v->d_mix_scratch && (e = cudaMalloc(&v->d_mix_scratch, (size_t)C * B * sizeof(float))) != cudaSuccess) return e;
  if (!v->d_mix_table) {
    if ((e = cudaMalloc(&v->d_mix_table, (size_t)(4 * C + 1) * sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(v->d_mix_table, 0, (size_t)(4 * C + 1) * sizeof(int), v->stream)) != cudaSuccess)
      return e;
  }
  if (!v->h_clip && (e = cudaHostAlloc(reinterpret_cast<void**>(&v->h_clip), sizeof(int), cudaHostAllocMapped)) !=
                        cudaSuccess)
    return e;
  int* chan_group = v->d_mix_table;
  int* gstart = chan_group + C;
  int* gchan = gstart + C + 1;
  unsigned* count = reinterpret_cast<unsigned*>(gchan + C);
  std::vector<uint32_t> map(pcm.group, pcm.group + C);
  map.push_back(pcm.ngroups);
  if (map != v->mix_groups) {
    std::vector<int> t(3 * C + 1);
    int* hg = t.data();
    int* hs = hg + C;
    int* hc = hs + C + 1;
    std::vector<int> fill(pcm.ngroups + 1, 0);
    for (int c = 0; c < C; ++c) {
      hg[c] = (int)pcm.group[c];
      fill[pcm.group[c] + 1] += 1;
    }
    for (uint32_t g = 0; g < pcm.ngroups; ++g) fill[g + 1] += fill[g];
    for (uint32_t g = 0; g <= pcm.ngroups; ++g) hs[g] = fill[g];
    for (int c = 0; c < C; ++c) hc[fill[pcm.group[c]]++] = c;  // ascending within each group
    if ((e = cudaMemcpyAsync(chan_group, hg, t.size() * sizeof(int), cudaMemcpyHostToDevice, v->stream)) !=
        cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(v->stream)) != cudaSuccess) return e;  // t is pageable and local
    v->mix_groups = map;
  }
  epi->active = 1;
  epi->in_scale = pcm.in_gain / 32767;
  epi->out_scale = 32767 * pcm.out_gain;
  epi->chan_group = chan_group;
  epi->gstart = gstart;
  epi->gchan = gchan;
  epi->count = count;
  epi->scratch = v->d_mix_scratch;
  epi->clip = v->h_clip;
  return cudaSuccess;
}

int32_t process_common(tanb_convolution* v, Mem in_mem, const float* const* in, Mem out_mem, float* const* out,
                       size_t n, const uint32_t* flags, size_t* done, const PcmIO* pcm = nullptr) {
  tanb::NvtxRange range("tanb Process");
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (done) *done = 0;
  if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "Process before Init");
  if (!in) return fail(TANB_INVALID_ARG, "ppBufferInput == NULL");
  if (!out) return fail(TANB_INVALID_ARG, "ppBufferOutput == NULL");
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  if (v->td) return td_process(v, in_mem, in, out_mem, out, n, flags, done);
  if (v->nu_eng) {
    if (pcm) return fail(TANB_NOT_SUPPORTED, "the fused PCM pipeline runs the uniformly partitioned methods");
    return nu_process(v, in_mem, in, out_mem, out, n, flags, done);
  }
  if (run_pending_finalize(v) != TANB_OK) return TANB_FAIL;

  const int B = v->B, C = v->C, P = v->P;
  size_t nblocks = n / (size_t)B;
  size_t processed = 0;
  int32_t status = TANB_OK;
  tanb::MixEpi epi;
  if (pcm) {
    TANB_CUDA(ensure_mix(v, *pcm, &epi));
    *v->h_clip = 0;
  }
  std::vector<uint8_t>& run = v->scr_run;
  std::vector<uint8_t>& flush = v->scr_flush;
  std::vector<std::vector<uint8_t>>& run_b = v->scr_run_b;
  std::vector<std::vector<int>>& flush_b = v->scr_flush_b;
  std::vector<int>& cur_b = v->scr_cur_b;

  const bool param = C <= tanb::kParamChannels;
  // rows in the object's staging (host rows, the fused pipeline's int16 rows
  // and its scratch outputs): two base pointers describe every channel
  const bool staged = param && (pcm || (in_mem == Mem::Host && out_mem == Mem::Host));
  const bool host_out = out_mem == Mem::Host;  // the call returns once the heads have signalled
  // Caller rows the kernels can address in place (pinned host memory), on
  // calls that wait for the heads anyway, so that the caller's rows are free
  // again when the call returns.
  PinnedRows pin_in, pin_out;
  bool direct_in = staged && !pcm && pinned_rows(in, C, n, true, &pin_in);
  bool direct_out = staged && !pcm && pinned_rows(out, C, n, false, &pin_out);
  if (direct_in && direct_out && pin_in.lo < pin_out.hi && pin_out.lo < pin_in.hi)
    direct_in = direct_out = false;  // in place or aliased: staging keeps the reads before the writes
  using Clock = std::chrono::steady_clock;
  auto us = [](Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::micro>(b - a).count();
  };
  const Clock::time_point t_call = Clock::now();
  double t_stage = 0, t_launch = 0, t_wait = 0, t_copy = 0;
  while (processed < nblocks && status == TANB_OK) {
    const Clock::time_point t0 = Clock::now();
    int nb = (int)std::min<size_t>(kMaxBlocksPerChunk, nblocks - processed);
    TANB_CUDA(cudaEventSynchronize(v->ev_stage));
    if (v->staging_busy) {
      TANB_CUDA(cudaEventSynchronize(v->ev_out));
      v->staging_busy = false;
    }
    int filled = 0;
    for (int b = 0; b < nb; ++b) {
      const size_t blk = processed + b;
      int nrun = channel_flags(v, flags, run, flush);
      if (nrun == 0) {
        status = fail(TANB_WRONG_STATE, "no running channels");
        break;
      }
      tanb::ParamDesc* pd = param ? &v->pdesc[b] : nullptr;
      tanb::StageDesc* sd = staged ? &v->sdesc[b] : nullptr;
      ChanCtl* ctl = param ? nullptr : v->desc_ctl(v->h_stage, b);
      const float** din = param ? nullptr : v->desc_in(v->h_stage, b);
      float** dout = param ? nullptr : v->desc_out(v->h_stage, b);
      flush_b[b].clear();
      for (int c = 0; c < C; ++c) {
        if (flush[c]) flush_b[b].push_back(c);
        const int sw = (v->pending[c] && run[c]) ? 1 : 0;
        const ChanCtl cc{run[c], sw, v->active[c], v->slot_new[c]};
        const float* x = nullptr;
        float* y = nullptr;
        if (sw) {
          v->active[c] = v->slot_new[c];
          v->pending[c] = 0;
        }
        // A null row reads as silence and its output is discarded. Host rows
        // go through pinned staging that the head kernel reads and writes in
        // place (mapped host memory under unified addressing): no separate
        // host<->device copies per block.
        if (pcm) {
          // int16 samples, converted by the head kernel as it loads them
          int16_t* row = reinterpret_cast<int16_t*>(v->stage_in(v->h_stage, b, c));
          const int16_t* src = pcm->in[c] + blk * B * pcm->in_step;
          for (int i = 0; i < B; ++i) row[i] = src[(size_t)i * pcm->in_step];
          x = v->stage_in(v->h_stage, b, c);
        } else if (in_mem == Mem::Host && direct_in) {
          x = in[c] ? in[c] + blk * B : nullptr;
        } else if (in_mem == Mem::Host) {
          x = in[c] ? v->stage_in(v->h_stage, b, c) : nullptr;
          if (run[c] && in[c])
            tanb::copy_rows_for_device(v->stage_in(v->h_stage, b, c), in[c] + blk * B, B * sizeof(float));
        } else {
          x = in[c] ? in[c] + blk * B : nullptr;
        }
        if (pcm) {
          y = v->d_mix_scratch + (size_t)c * B;
        } else if (direct_out) {
          y = out[c] + blk * B;
        } else if (out_mem == Mem::Host) {
          y = v->h_out + ((size_t)b * C + c) * B;
        } else {
          y = out[c] ? out[c] + blk * B : nullptr;
        }
        if (sd) {
          sd->c.ctl[c] = tanb::pack_ctl(cc, x != nullptr);
        } else if (pd) {
          pd->c.ctl[c] = tanb::pack_ctl(cc, x != nullptr);
          pd->in[c] = x;
          pd->out[c] = y;
        } else {
          ctl[c] = cc;
          din[c] = x;
          dout[c] = y;
        }
      }
      if (sd) {
        if (direct_in) {
          sd->in = pin_in.base + blk * B;
          sd->stride = pin_in.stride;
        } else {
          sd->in = v->stage_in(v->h_stage, b, 0);
          sd->stride = B;
        }
        if (direct_out) {
          sd->out = const_cast<float*>(pin_out.base) + blk * B;
          sd->ostride = pin_out.stride;
        } else {
          sd->out = pcm ? v->d_mix_scratch : v->h_out + (size_t)b * C * B;
          sd->ostride = B;
        }
      }
      run_b[b] = run;
      v->cur = (v->cur - 1 + P) % P;
      cur_b[b] = v->cur;
      ++filled;
    }
    nb = filled;
    if (nb == 0) break;
    tanb::copy_for_device_fence();  // staged rows are visible before the launches
    const Clock::time_point t1 = Clock::now();
    t_stage += us(t0, t1);
    // ev_stage guards the host descriptor tables until their upload has run;
    // ev_out guards the host staging rows until the heads have read and
    // written them. A call on device rows with parameter descriptors uses
    // neither and records no event.
    if (!param) {
      TANB_CUDA(cudaMemcpyAsync(v->d_stage, v->h_stage, nb * v->desc_bytes, cudaMemcpyHostToDevice, v->stream));
      TANB_CUDA(cudaEventRecord(v->ev_stage, v->stream));
    }
    for (int b = 0; b < nb; ++b) {
      for (int c : flush_b[b]) TANB_CUDA(flush_channel(v, c));
      const ChanCtl* dctl = v->desc_ctl(v->d_stage, b);
      tanb::BlockRef ref;
      if (staged) {
        ref.stage = &v->sdesc[b];
      } else if (param) {
        ref.param = &v->pdesc[b];
      } else {
        ref.ctl = dctl;
        ref.in = v->desc_in(v->d_stage, b);
        ref.out = v->desc_out(v->d_stage, b);
      }
      if (pcm) epi.out16 = reinterpret_cast<int16_t*>(v->h_out + (size_t)b * C * B);  // [ngroups][B] of block b
      const int parity = (int)((v->blocks + b) & 1);
      tanb::HeadSignal sig;
      if (host_out) sig = tanb::HeadSignal{v->d_head_count, v->d_head_flag, ++v->head_seq};
      TANB_CUDA(counted(v, tanb_convolution::kHead,
                        [&] { return tanb::launch_head(v->ds, ref, cur_b[b], parity, v->stream, epi, sig); }));
      const bool last = (b == nb - 1);
      if (last) {
        v->last_desc = dctl;
        v->last_is_param = param;
        if (param) v->last_ctlp = staged ? v->sdesc[b].c : v->pdesc[b].c;
        v->last_cur = cur_b[b];
      }
      if (last && v->finalize_mode) {
        v->finalize_due = true;
      } else if (P > 2) {
        // Directly behind the head (programmatic serialization): the next
        // block's partitions >= 2 share no data with this head, so the two run
        // side by side.
        TANB_CUDA(counted(v, tanb_convolution::kTail, [&] {
          return tanb::launch_tail(v->ds, ref, 0, cur_b[b], parity ^ 1, v->tiling, v->stream, true);
        }));
      }
    }
    // Outputs are final after the heads; in the default mode the last tail,
    // which overlaps its head, completes before this event as well. The
    // staged inputs and outputs are free again once it has completed.
    if (pcm || in_mem == Mem::Host || out_mem == Mem::Host) {
      TANB_CUDA(cudaEventRecord(v->ev_out, v->stream));
      v->staging_busy = true;
    }
    const Clock::time_point t2 = Clock::now();
    t_launch += us(t1, t2);
    if (host_out) {
      // the outputs are final once the last head has signalled; the tail
      // launched behind it keeps running while they are scattered
      if (wait_heads(v, v->head_seq) != TANB_OK) return TANB_FAIL;
      const Clock::time_point t3 = Clock::now();
      t_wait += us(t2, t3);
      v->staging_busy = false;
      if (*v->h_err != tanb::kErrNone) return fail(TANB_FAIL, "device wait timed out (error %d)", *v->h_err);
      if (pcm) {
        for (int b = 0; b < nb; ++b) {
          const int16_t* st = reinterpret_cast<const int16_t*>(v->h_out + (size_t)b * C * B);
          for (uint32_t g = 0; g < pcm->ngroups; ++g) {
            int16_t* dst = pcm->out[g] + (processed + b) * B * pcm->out_step;
            for (int i = 0; i < B; ++i) dst[(size_t)i * pcm->out_step] = st[(size_t)g * B + i];
          }
        }
      } else if (!direct_out) {
        for (int b = 0; b < nb; ++b)
          for (int c = 0; c < C; ++c)
            if (run_b[b][c] && out[c])
              std::memcpy(out[c] + (processed + b) * B, v->h_out + ((size_t)b * C + c) * B, B * sizeof(float));
      }
      t_copy += us(t3, Clock::now());
    }
    processed += nb;
    v->blocks += nb;
    if (v->finalize_mode && processed < nblocks && status == TANB_OK) {
      if (run_pending_finalize(v) != TANB_OK) return TANB_FAIL;
    }
  }
  if (done) *done = processed * B;
  v->ct[0] = t_stage;
  v->ct[1] = t_launch;
  v->ct[2] = t_wait;
  v->ct[3] = t_copy;
  v->ct[4] = us(t_call, Clock::now());
  v->ct[5] = (direct_in ? 1 : 0) + (direct_out ? 2 : 0);
  return status;
}

// ---------------------------------------------------------------------------
// Non-uniform methods (TANB_METHOD_FFT_PARTITIONED_NONUNIFORM and the FHT / FFT
// NONUNIFORM_PARTITIONED GPU names; the reference's CPU form is
// ConvolutionImpl.cpp:224-246, 2416-2428), on a private engine session.
// ---------------------------------------------------------------------------

constexpr int kNuBlocksPerChunk = kMaxBlocksPerChunk;

// The default level schedule for an IR of L taps at block B: two partitions per
// size, doubling from B up to about L / 16 (at most 16384), the largest size
// taking the rest (tanb_nu_schedule).
int32_t nu_default_schedule(uint32_t L, uint32_t B, std::vector<uint32_t>* blocks, std::vector<uint32_t>* parts) {
  uint32_t mx = B;
  while (mx < 16384 && (uint64_t)mx * 32 <= L) mx <<= 1;
  uint32_t nl = 0;
  blocks->assign(16, 0);
  parts->assign(16, 0);
  const int32_t r = tanb_nu_schedule(L, B, mx, &nl, blocks->data(), parts->data());
  blocks->resize(nl);
  parts->resize(nl);
  return r;
}

int32_t nu_init(tanb_convolution* v, uint32_t L, uint32_t B, uint32_t C, uint32_t nlevels, const uint32_t* blocks,
                const uint32_t* parts) {
  if (B < 128 || B > 2048)
    return fail(TANB_NOT_SUPPORTED, "the non-uniform methods run blocks in [128, 2048] (block %u)", B);
  if (nlevels) {
    v->nu_blocks.assign(blocks, blocks + nlevels);
    v->nu_parts.assign(parts, parts + nlevels);
  } else if (nu_default_schedule(L, B, &v->nu_blocks, &v->nu_parts) != TANB_OK) {
    return TANB_INVALID_ARG;
  }
  const uint32_t nl = (uint32_t)v->nu_blocks.size();
  const size_t bytes = tanb::engine_nu_session_bytes((int)B, TANB_SPECTRUM_FP32, (int)C, L, nl, v->nu_blocks.data(),
                                                     v->nu_parts.data());
  if (!bytes) return fail(TANB_INVALID_ARG, "invalid non-uniform level schedule");
  int32_t r = tanb_engine_create(v->ctx, B, TANB_SPECTRUM_FP32, bytes, C, 0, &v->nu_eng);
  if (r != TANB_OK) return r;
  uint32_t first = 0;
  r = tanb_engine_open_session_nu(v->nu_eng, C, L, nl, v->nu_blocks.data(), v->nu_parts.data(), &v->nu_sess, &first);
  if (r == TANB_OK) r = tanb_engine_io(v->nu_eng, &v->nu_in, &v->nu_out);
  if (r != TANB_OK) {
    const std::string msg = tanb_last_error();
    free_all(v);
    return fail(r, "%s", msg.c_str());
  }
  const size_t tab = (size_t)kNuBlocksPerChunk * 2 * C * sizeof(float*);
  cudaError_t e = cudaMallocHost(&v->h_nu_tab, tab);
  if (e == cudaSuccess) e = cudaMalloc(&v->d_nu_tab, tab);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&v->ev_stage, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(v->ev_stage, (cudaStream_t)tanb_engine_stream(v->nu_eng));
  if (e != cudaSuccess) {
    free_all(v);
    return fail(e == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "non-uniform setup: %s",
                cudaGetErrorString(e));
  }
  int64_t info[8];
  tanb_engine_info(v->nu_eng, info);
  v->dev_bytes = (size_t)info[4];
  return TANB_OK;
}

// UpdateResponseTD: channels flagged STOP_INPUT keep their IR, FLUSH_STREAM
// channels are flushed; the transform completes before this returns, so the
// new IR takes effect (with the one-block crossfade) on the next block.
int32_t nu_update(tanb_convolution* v, Mem mem, const float* const* ir, size_t n, const uint32_t* flags) {
  const int C = v->C;
  std::vector<uint8_t> mask(C, 1);
  for (int c = 0; c < C; ++c) {
    if (flags && (flags[c] & kFlush)) {
      const int32_t r = tanb::engine_flush_channel(v->nu_eng, v->nu_sess, c);
      if (r != TANB_OK) return r;
    }
    if (flags && (flags[c] & kStopInput)) mask[c] = 0;
  }
  return tanb::engine_update_channels(v->nu_eng, v->nu_sess, ir, n, mem == Mem::Device,
                                      TANB_OPERATION_FLAG_BLOCK_UNTIL_READY, mask.data());
}

int32_t nu_process(tanb_convolution* v, Mem in_mem, const float* const* in, Mem out_mem, float* const* out,
                   size_t n, const uint32_t* flags, size_t* done) {
  const int B = v->B, C = v->C;
  const size_t nblocks = n / (size_t)B;
  cudaStream_t st = (cudaStream_t)tanb_engine_stream(v->nu_eng);
  // Host rows go through the engine's pinned rows, one block at a time (its
  // graph when both sides are host rows); device rows through row tables,
  // written for a chunk of blocks and uploaded once before the chunk's blocks.
  const bool host_io = in_mem == Mem::Host || out_mem == Mem::Host;
  const bool tables = in_mem == Mem::Device || out_mem == Mem::Device;
  size_t processed = 0;
  int32_t status = TANB_OK;
  while (processed < nblocks && status == TANB_OK) {
    const int nb = host_io ? 1 : (int)std::min<size_t>(kNuBlocksPerChunk, nblocks - processed);
    TANB_CUDA(cudaEventSynchronize(v->ev_stage));  // the previous chunk's tables have been uploaded
    // pass 1: channel flags of every block of the chunk and its row tables
    int filled = 0;
    for (int b = 0; b < nb; ++b) {
      std::vector<uint8_t>& run = v->scr_run_b[b];
      if (channel_flags(v, flags, run, v->scr_flush) == 0) {
        status = fail(TANB_WRONG_STATE, "no running channels");
        break;
      }
      v->scr_flush_b[b].clear();
      for (int c = 0; c < C; ++c)
        if (v->scr_flush[c]) v->scr_flush_b[b].push_back(c);
      const size_t blk = processed + b;
      const float** tin = v->h_nu_tab + (size_t)(2 * b) * C;
      const float** tout = tin + C;
      for (int c = 0; c < C; ++c) {
        if (in_mem == Mem::Device) tin[c] = (run[c] && in[c]) ? in[c] + blk * B : nullptr;
        if (out_mem == Mem::Device) tout[c] = (run[c] && out[c]) ? out[c] + blk * B : nullptr;
      }
      ++filled;
    }
    if (filled && tables)
      TANB_CUDA(cudaMemcpyAsync(v->d_nu_tab, v->h_nu_tab, (size_t)2 * filled * C * sizeof(float*),
                                cudaMemcpyHostToDevice, st));
    // pass 2: flushes (ordered on the engine's stream before the block), input
    // rows, the block, output rows
    for (int b = 0; b < filled; ++b) {
      const size_t blk = processed + b;
      const std::vector<uint8_t>& run = v->scr_run_b[b];
      for (int c : v->scr_flush_b[b]) {
        const int32_t r = tanb::engine_flush_channel(v->nu_eng, v->nu_sess, c);
        if (r != TANB_OK) return r;
      }
      tanb::EngRows rows;
      rows.ld = B;
      if (in_mem == Mem::Host) {
        // free channels and missing rows read silence
        for (int c = 0; c < C; ++c) {
          float* row = v->nu_in + (size_t)c * B;
          if (run[c] && in[c])
            tanb::copy_rows_for_device(row, in[c] + blk * B, B * sizeof(float));
          else
            std::memset(row, 0, B * sizeof(float));
        }
        tanb::copy_for_device_fence();
        rows.in_base = v->nu_in;
      } else {
        rows.in_tab = v->d_nu_tab + (size_t)(2 * b) * C;
      }
      if (out_mem == Mem::Host)
        rows.out_base = v->nu_out;
      else
        rows.out_tab = reinterpret_cast<float* const*>(const_cast<float**>(v->d_nu_tab + (size_t)(2 * b + 1) * C));
      int32_t r;
      if (in_mem == Mem::Host && out_mem == Mem::Host) {
        r = tanb_engine_process(v->nu_eng);  // the engine's graph over its pinned rows; waits for the output
      } else {
        r = tanb::engine_process_rows(v->nu_eng, rows);
        if (r == TANB_OK && host_io) TANB_CUDA(cudaStreamSynchronize(st));  // pinned rows reused next block
      }
      if (r != TANB_OK) return r;
      if (out_mem == Mem::Host)
        for (int c = 0; c < C; ++c)
          if (run[c] && out[c]) std::memcpy(out[c] + blk * B, v->nu_out + (size_t)c * B, B * sizeof(float));
    }
    if (tables) TANB_CUDA(cudaEventRecord(v->ev_stage, st));
    processed += filled;
    v->blocks += filled;
  }
  if (done) *done = processed * B;
  return status;
}

// ---------------------------------------------------------------------------
// TIME_DOMAIN method (ConvolutionImpl.cpp:407-468, 721-762, 2645-2782)
// ---------------------------------------------------------------------------

cudaError_t td_alloc(tanb_convolution* v) {
  const size_t C = v->C, len = v->length;
  cudaError_t e;
  if ((e = dev_alloc(v, &v->td_hist, C * len)) != cudaSuccess) return e;
  if ((e = dev_alloc(v, &v->td_ir, 2 * C * len)) != cudaSuccess) return e;
  if ((e = dev_alloc(v, &v->td_dir, C * len)) != cudaSuccess) return e;
  if ((e = dev_alloc(v, &v->td_io, 2 * C * len)) != cudaSuccess) return e;
  if ((e = dev_alloc(v, &v->d_tdchan, C)) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&v->h_td, 3 * C * len * sizeof(float))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&v->h_tdchan, C * sizeof(tanb::TdChan))) != cudaSuccess) return e;
  v->td_pos.assign(C, 0);
  v->td_fade = -1;
  v->td_swapping.assign(C, 0);
  return cudaSuccess;
}

float* td_ir_row(tanb_convolution* v, int slot, int c) {
  return v->td_ir + ((size_t)slot * v->C + c) * v->length;
}

int32_t td_update(tanb_convolution* v, Mem mem, const float* const* ir, size_t n, const uint32_t* flags,
                  uint32_t op) {
  const size_t len = v->length;
  TANB_CUDA(cudaStreamSynchronize(v->stream));  // pinned IR staging is reused
  for (int c = 0; c < v->C; ++c) {
    if (flags && (flags[c] & kFlush)) {
      TANB_CUDA(cudaMemsetAsync(v->td_hist + (size_t)c * len, 0, len * sizeof(float), v->stream));
      v->td_pos[c] = 0;
    }
    if (flags && (flags[c] & kStopInput)) continue;
    if (!ir[c] && n > 0) return fail(TANB_INVALID_ARG, "ppBuffer[%d] == NULL", c);
    if (!v->pending[c]) {
      v->slot_new[c] = 1 - v->active[c];
      v->pending[c] = 1;
    }
    float* dst = td_ir_row(v, v->slot_new[c], c);
    if (mem == Mem::Host) {
      float* row = v->h_td + (size_t)c * len;
      if (n) tanb::copy_for_device(row, ir[c], n * sizeof(float));
      std::memset(row + n, 0, (len - n) * sizeof(float));
      TANB_CUDA(cudaMemcpyAsync(dst, row, len * sizeof(float), cudaMemcpyHostToDevice, v->stream));
    } else {
      if (n) TANB_CUDA(cudaMemcpyAsync(dst, ir[c], n * sizeof(float), cudaMemcpyDeviceToDevice, v->stream));
      TANB_CUDA(cudaMemsetAsync(dst + n, 0, (len - n) * sizeof(float), v->stream));
    }
  }
  if (op & TANB_OPERATION_FLAG_BLOCK_UNTIL_READY) TANB_CUDA(cudaStreamSynchronize(v->stream));
  return TANB_OK;
}

// Runs one TIME_DOMAIN call: the descriptors in h_tdchan are filled; inputs
// are staged (host) or referenced (device); outputs go to staging (host).
int32_t td_launch(tanb_convolution* v, int n, bool host_in, bool host_out, float* const* out) {
  const size_t C = v->C, len = v->length;
  float* h_in = v->h_td + C * len;
  float* h_out = v->h_td + 2 * C * len;
  if (host_in)
    TANB_CUDA(cudaMemcpyAsync(v->td_io, h_in, C * len * sizeof(float), cudaMemcpyHostToDevice, v->stream));
  TANB_CUDA(cudaMemcpyAsync(v->d_tdchan, v->h_tdchan, C * sizeof(tanb::TdChan), cudaMemcpyHostToDevice,
                            v->stream));
  TANB_CUDA(counted(v, tanb_convolution::kTail,
                    [&] { return tanb::launch_td(v->td_hist, (int)len, v->d_tdchan, (int)C, n, v->B, v->stream); }));
  if (host_out) {
    TANB_CUDA(cudaMemcpyAsync(h_out, v->td_io + C * len, C * len * sizeof(float), cudaMemcpyDeviceToHost,
                              v->stream));
  }
  TANB_CUDA(cudaStreamSynchronize(v->stream));
  if (host_out)
    for (size_t c = 0; c < C; ++c)
      if (v->h_tdchan[c].run && out[c]) std::memcpy(out[c], h_out + c * len, n * sizeof(float));
  return TANB_OK;
}

int32_t td_process(tanb_convolution* v, Mem in_mem, const float* const* in, Mem out_mem, float* const* out,
                   size_t n, const uint32_t* flags, size_t* done) {
  const size_t C = v->C, len = v->length;
  const int ns = (int)std::min<size_t>(n, (size_t)v->B);
  if (ns == 0) return TANB_OK;
  std::vector<uint8_t> run(C), flush(C);
  if (channel_flags(v, flags, run, flush) == 0) return fail(TANB_WRONG_STATE, "no running channels");
  TANB_CUDA(cudaStreamSynchronize(v->stream));
  for (size_t c = 0; c < C; ++c)
    if (flush[c]) {
      TANB_CUDA(cudaMemsetAsync(v->td_hist + c * len, 0, len * sizeof(float), v->stream));
      v->td_pos[c] = 0;
    }
  if (v->td_fade < 0) {
    bool any = false;
    for (size_t c = 0; c < C; ++c) {
      v->td_swapping[c] = v->pending[c] && run[c];
      any = any || v->td_swapping[c];
    }
    if (any) v->td_fade = 0;
  }
  float* h_in = v->h_td + C * len;
  for (size_t c = 0; c < C; ++c) {
    tanb::TdChan& t = v->h_tdchan[c];
    t = tanb::TdChan{};
    t.run = run[c];
    t.pos = v->td_pos[c];
    t.first = 0;
    t.last = (int)len;
    t.ir = td_ir_row(v, v->active[c], c);
    t.ir_new = td_ir_row(v, v->slot_new[c], c);
    t.swap = (v->td_fade >= 0 && v->td_swapping[c]) ? 1 : 0;
    t.fade0 = v->td_fade < 0 ? 0 : v->td_fade;
    if (in_mem == Mem::Host) {
      t.in = in[c] ? v->td_io + c * len : nullptr;
      if (in[c] && run[c]) tanb::copy_for_device(h_in + c * len, in[c], ns * sizeof(float));
    } else {
      t.in = in[c];
    }
    t.out = out_mem == Mem::Host ? v->td_io + (C + c) * len : out[c];
  }
  int32_t r = td_launch(v, ns, in_mem == Mem::Host, out_mem == Mem::Host, out);
  if (r != TANB_OK) return r;
  for (size_t c = 0; c < C; ++c)
    if (run[c]) v->td_pos[c] = (int)((v->td_pos[c] + ns) % len);
  if (v->td_fade >= 0) {
    v->td_fade += ns;
    if (v->td_fade >= v->B) {
      for (size_t c = 0; c < C; ++c)
        if (v->td_swapping[c]) {
          v->active[c] = v->slot_new[c];
          v->pending[c] = 0;
          v->td_swapping[c] = 0;
        }
      v->td_fade = -1;
    }
  }
  if (done) *done = ns;
  return TANB_OK;
}

int32_t td_process_direct(tanb_convolution* v, const float* const* ir, const float* const* in, float* const* out,
                          size_t n, size_t* done, const int32_t* nz) {
  const size_t C = v->C, len = v->length;
  if (n > len) n = len;
  for (size_t c = 0; c < C; ++c) {
    const int first = nz ? nz[2 * c] : 0, last = nz ? nz[2 * c + 1] : (int)len;
    if (first < 0 || last > (int)len || first > last)
      return fail(TANB_INVALID_ARG, "nzFirstLast[%zu] = [%d, %d) outside [0, %zu]", c, first, last, len);
    if (!in[c] || !out[c] || (!ir[c] && last > first)) return fail(TANB_INVALID_ARG, "null buffer for channel %zu", c);
  }
  if (n == 0) return TANB_OK;
  TANB_CUDA(cudaStreamSynchronize(v->stream));
  float* h_in = v->h_td + C * len;
  for (size_t c = 0; c < C; ++c) {
    const int first = nz ? nz[2 * c] : 0, last = nz ? nz[2 * c + 1] : (int)len;
    float* row = v->h_td + c * len;
    if (last > first) {
      tanb::copy_for_device(row + first, ir[c] + first, (last - first) * sizeof(float));
      TANB_CUDA(cudaMemcpyAsync(v->td_dir + c * len + first, row + first, (last - first) * sizeof(float),
                                cudaMemcpyHostToDevice, v->stream));
    }
    tanb::copy_for_device(h_in + c * len, in[c], n * sizeof(float));
    tanb::TdChan& t = v->h_tdchan[c];
    t = tanb::TdChan{};
    t.run = 1;
    t.pos = v->td_pos[c];
    t.first = first;
    t.last = last;
    t.ir = v->td_dir + c * len;
    t.in = v->td_io + c * len;
    t.out = v->td_io + (C + c) * len;
  }
  int32_t r = td_launch(v, (int)n, true, true, out);
  if (r != TANB_OK) return r;
  for (size_t c = 0; c < C; ++c) v->td_pos[c] = (int)((v->td_pos[c] + n) % len);
  if (done) *done = n;
  return TANB_OK;
}

}  // namespace

extern "C" {

const char* tanb_last_error(void) { return g_last_error.c_str(); }

int32_t tanb_create_context(uint64_t version, int32_t device, tanb_context** ctx) {
  if (!ctx) return fail(TANB_INVALID_POINTER, "ppContext == NULL");
  *ctx = nullptr;
  if ((version >> 48) != 1) return fail(TANB_TAN_UNSUPPORTED_VERSION, "unsupported version %llu", (unsigned long long)(version >> 48));
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(TANB_NO_DEVICE, "no CUDA device available");
  if (device < 0 || device >= count) return fail(TANB_INVALID_ARG, "device %d out of range", device);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return fail(TANB_NO_DEVICE, "device query failed");
  if (prop.major != 10) return fail(TANB_NO_DEVICE, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
  tanb_context* c = new tanb_context();
  c->device = device;
  *ctx = c;
  return TANB_OK;
}

int32_t tanb_context_release(tanb_context* ctx) {
  delete ctx;
  return TANB_OK;
}

int32_t tanb_create_convolution(tanb_context* ctx, tanb_convolution** conv) {
  if (!ctx) return fail(TANB_INVALID_POINTER, "pContext == NULL");
  if (!conv) return fail(TANB_INVALID_POINTER, "ppConvolution == NULL");
  tanb_convolution* v = new tanb_convolution();
  v->ctx = ctx;
  *conv = v;
  return TANB_OK;
}

int32_t tanb_convolution_terminate(tanb_convolution* v) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (v->initialized) cudaSetDevice(v->ctx->device);
  free_all(v);
  v->initialized = false;
  v->terminated = true;
  return TANB_OK;
}

int32_t tanb_convolution_release(tanb_convolution* v) {
  if (!v) return TANB_OK;
  tanb_convolution_terminate(v);
  delete v;
  return TANB_OK;
}

}  // extern "C"

namespace {

int32_t init_impl(tanb_convolution* v, uint32_t method, uint32_t L, uint32_t B, uint32_t C, uint32_t nlevels,
                  const uint32_t* level_block, const uint32_t* level_parts) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (v->terminated) return fail(TANB_WRONG_STATE, "Cannot initialize after termination");
  if (L == 0) return fail(TANB_INVALID_ARG, "lengthInSamples == 0");
  if (B == 0) return fail(TANB_INVALID_ARG, "bufferSizeInSamples == 0");
  if (C == 0) return fail(TANB_INVALID_ARG, "channels == 0");
  if ((B & (B - 1)) != 0) return fail(TANB_INVALID_ARG, "bufferSizeInSamples must be power of 2");
  if (B < 32 || B > 8192) return fail(TANB_INVALID_ARG, "bufferSizeInSamples must be in [32, 8192]");
  if (v->initialized) return fail(TANB_ALREADY_INITIALIZED, "Already initialized");
  const uint32_t extra = method & 0xC000u;
  const uint32_t base = method & ~0xC000u;
  if (base > TANB_METHOD_FFT_NONUNIFORM_PARTITIONED) return fail(TANB_NOT_SUPPORTED, "convolutionMethod isn't supported");
  v->method = base;
  v->finalize_mode = (extra == TANB_METHOD_USE_PROCESS_FINALIZE);
  v->finalize_due = false;
  v->L = (int)L;
  v->B = (int)B;
  v->C = (int)C;
  v->P = (int)((L + B - 1) / B);
  if (v->P < 1) v->P = 1;
  int len = 1;
  while ((uint32_t)len < L) len <<= 1;
  v->length = len;
  int log2B = 0;
  while ((1 << log2B) < (int)B) ++log2B;

  cudaError_t e = cudaSetDevice(v->ctx->device);
  if (e != cudaSuccess) return fail(TANB_NO_DEVICE, "cudaSetDevice: %s", cudaGetErrorString(e));
  auto host_state = [&] {
    v->active.assign(C, 0);
    v->pending.assign(C, 0);
    v->slot_new.assign(C, 1);
    v->tail_left.assign(C, 0);
    v->available.assign(C, 0);
    v->flushed.assign(C, 0);
    v->scr_run.assign(C, 0);
    v->scr_flush.assign(C, 0);
    v->scr_run_b.assign(kMaxBlocksPerChunk, std::vector<uint8_t>(C, 0));
    v->scr_flush_b.assign(kMaxBlocksPerChunk, std::vector<int>());
    for (auto& f : v->scr_flush_b) f.reserve(C);
    v->scr_cur_b.assign(kMaxBlocksPerChunk, 0);
    v->cur = 0;
    v->blocks = 0;
  };
  const bool nonuniform = base == TANB_METHOD_FFT_PARTITIONED_NONUNIFORM ||
                          base == TANB_METHOD_FHT_NONUNIFORM_PARTITIONED ||
                          base == TANB_METHOD_FFT_NONUNIFORM_PARTITIONED;
  if (nonuniform) {
    const int32_t r = nu_init(v, L, B, C, nlevels, level_block, level_parts);
    if (r != TANB_OK) return r;
    v->finalize_mode = false;  // the head and every level run in one graph launch per block
    host_state();
    v->initialized = true;
    return TANB_OK;
  }
  if (nlevels) return fail(TANB_INVALID_ARG, "a level schedule needs a non-uniform method");
  if ((e = tanb::prepare_kernels()) != cudaSuccess) return fail(TANB_FAIL, "kernel setup: %s", cudaGetErrorString(e));
  if ((e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(TANB_FAIL, "stream: %s", cudaGetErrorString(e));
  const size_t Cs = C, Bs = B, Ps = v->P;
  v->td = (base == TANB_METHOD_TIME_DOMAIN);
  if (v->td) {
    e = td_alloc(v);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
    if (e != cudaSuccess) {
      free_all(v);
      cudaGetLastError();
      return fail(e == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "allocation failed: %s",
                  cudaGetErrorString(e));
    }
    v->active.assign(C, 0);
    v->pending.assign(C, 0);
    v->slot_new.assign(C, 1);
    v->tail_left.assign(C, 0);
    v->available.assign(C, 0);
    v->flushed.assign(C, 0);
    v->initialized = true;
    return TANB_OK;
  }
  v->desc_bytes = (sizeof(ChanCtl) + 2 * sizeof(void*)) * Cs;
  const size_t stage_bytes = kMaxBlocksPerChunk * (v->desc_bytes + Cs * Bs * sizeof(float));
  const size_t out_floats = kMaxBlocksPerChunk * Cs * Bs;

  do {
    if ((e = dev_alloc(v, &v->ds.H, Cs * 2 * Ps * Bs)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->ds.fdl, Cs * Ps * Bs)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->ds.prev, Cs * Bs)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->ds.tail, Cs * 3 * Bs)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->d_tw, 2 * Bs)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->d_stage, kMaxBlocksPerChunk * v->desc_bytes)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->d_head_count, 1)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->d_ir, Cs * Ps * Bs)) != cudaSuccess) break;
    if ((e = dev_alloc(v, &v->d_uctl, uctl_bytes(C))) != cudaSuccess) break;
    if ((e = cudaMallocHost(&v->h_stage, stage_bytes)) != cudaSuccess) break;
    if ((e = cudaMallocHost(&v->h_out, out_floats * sizeof(float))) != cudaSuccess) break;
    if ((e = cudaMallocHost(&v->h_ir, Cs * Ps * Bs * sizeof(float))) != cudaSuccess) break;
    if ((e = cudaMallocHost(&v->h_uctl, uctl_bytes(C))) != cudaSuccess) break;
    if ((e = cudaHostAlloc(&v->h_err, sizeof(int), cudaHostAllocMapped)) != cudaSuccess) break;
    if ((e = cudaHostAlloc(&v->h_head_flag, sizeof(long long), cudaHostAllocMapped)) != cudaSuccess) break;
    if ((e = cudaEventCreateWithFlags(&v->ev_stage, cudaEventDisableTiming)) != cudaSuccess) break;
    if ((e = cudaEventCreateWithFlags(&v->ev_ir, cudaEventDisableTiming)) != cudaSuccess) break;
    if ((e = cudaEventCreateWithFlags(&v->ev_out, cudaEventDisableTiming)) != cudaSuccess) break;
  } while (0);
  if (e != cudaSuccess) {
    free_all(v);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "allocation failed: %s",
                cudaGetErrorString(e));
  }
  std::memset(v->h_stage, 0, stage_bytes);
  std::vector<float2> tw(2 * Bs);
  tanb::make_twiddles(2 * B, tw.data());
  e = cudaMemcpyAsync(v->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, v->stream);
  if (e == cudaSuccess) e = cudaEventRecord(v->ev_stage, v->stream);
  if (e == cudaSuccess) e = cudaEventRecord(v->ev_ir, v->stream);
  if (e == cudaSuccess) e = cudaEventRecord(v->ev_out, v->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
  if (e != cudaSuccess) {
    free_all(v);
    return fail(TANB_FAIL, "init upload: %s", cudaGetErrorString(e));
  }
  v->ds.B = B;
  v->ds.log2B = log2B;
  v->ds.P = v->P;
  v->ds.C = C;
  v->ds.tw = v->d_tw;
  *v->h_err = tanb::kErrNone;
  *v->h_head_flag = 0;
  v->head_seq = 0;
  if ((e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&v->ds.err), v->h_err, 0)) != cudaSuccess ||
      (e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&v->d_head_flag), v->h_head_flag, 0)) != cudaSuccess) {
    free_all(v);
    return fail(TANB_FAIL, "mapped host words: %s", cudaGetErrorString(e));
  }
  v->tiling = default_tiling(B, v->P);
  host_state();
  v->pdesc.resize(C <= tanb::kParamChannels ? kMaxBlocksPerChunk : 0);
  v->sdesc.resize(C <= tanb::kParamChannels ? kMaxBlocksPerChunk : 0);
  v->initialized = true;
  return TANB_OK;
}

}  // namespace

extern "C" {

int32_t tanb_convolution_init(tanb_convolution* v, uint32_t method, uint32_t L, uint32_t B, uint32_t C) {
  return init_impl(v, method, L, B, C, 0, nullptr, nullptr);
}

int32_t tanb_convolution_init_nu(tanb_convolution* v, uint32_t method, uint32_t L, uint32_t B, uint32_t C,
                                 uint32_t nlevels, const uint32_t* level_block, const uint32_t* level_parts) {
  if (!level_block || !level_parts || nlevels == 0) return fail(TANB_INVALID_POINTER, "null level schedule");
  return init_impl(v, method, L, B, C, nlevels, level_block, level_parts);
}

int32_t tanb_convolution_update_response_td(tanb_convolution* v, const float* const* ir, size_t n,
                                            const uint32_t* flags, uint32_t op) {
  return update_common(v, Mem::Host, ir, n, flags, op);
}

int32_t tanb_convolution_update_response_td_device(tanb_convolution* v, const float* const* ir, size_t n,
                                                   const uint32_t* flags, uint32_t op) {
  return update_common(v, Mem::Device, ir, n, flags, op);
}

int32_t tanb_convolution_update_response_fd(tanb_convolution* v, const float* const*, size_t, const uint32_t*,
                                            uint32_t) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "not initialized");
  return fail(TANB_NOT_SUPPORTED, "UpdateResponseFD is not supported");
}

int32_t tanb_convolution_process(tanb_convolution* v, const float* const* in, float* const* out, size_t n,
                                 const uint32_t* flags, size_t* done) {
  return process_common(v, Mem::Host, in, Mem::Host, out, n, flags, done);
}

int32_t tanb_convolution_process_host_to_device(tanb_convolution* v, const float* const* in, float* const* out,
                                                size_t n, const uint32_t* flags, size_t* done) {
  int32_t r = process_common(v, Mem::Host, in, Mem::Device, out, n, flags, done);
  if (r == TANB_OK && v->initialized && !v->nu_eng) {
    cudaError_t e = cudaEventSynchronize(v->ev_out);
    if (e != cudaSuccess) return fail(TANB_FAIL, "sync: %s", cudaGetErrorString(e));
  }
  return r;
}

int32_t tanb_convolution_process_device(tanb_convolution* v, const float* const* in, float* const* out, size_t n,
                                        const uint32_t* flags, size_t* done) {
  return process_common(v, Mem::Device, in, Mem::Device, out, n, flags, done);
}

int32_t tanb_convolution_process_mix_pcm16(tanb_convolution* v, const int16_t* const* in, size_t in_step,
                                           float in_gain, const uint32_t* group, uint32_t ngroups,
                                           int16_t* const* out, size_t out_step, float out_gain, size_t n,
                                           int32_t* clipped, size_t* done) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  if (done) *done = 0;
  if (clipped) *clipped = 0;
  if (!in || !out || !group) return fail(TANB_INVALID_ARG, "null buffer or group map");
  if (!(in_gain > 0) || !(out_gain > 0)) return fail(TANB_INVALID_ARG, "conversion gains must be > 0");
  int C = 0;
  {
    std::lock_guard<std::mutex> lock(v->mu);
    if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "Process before Init");
    if (v->td || v->nu_eng)
      return fail(TANB_NOT_SUPPORTED, "the fused PCM pipeline runs the uniformly partitioned methods");
    C = v->C;
  }
  if (ngroups == 0 || ngroups > (uint32_t)C) return fail(TANB_INVALID_ARG, "ngroups must be in [1, channels]");
  std::vector<int> members(ngroups, 0);
  for (int c = 0; c < C; ++c) {
    if (!in[c]) return fail(TANB_INVALID_ARG, "input row %d == NULL", c);
    if (group[c] >= ngroups) return fail(TANB_INVALID_ARG, "group[%d] = %u out of range", c, group[c]);
    members[group[c]] += 1;
  }
  for (uint32_t g = 0; g < ngroups; ++g) {
    if (!out[g]) return fail(TANB_INVALID_ARG, "output row %u == NULL", g);
    if (!members[g]) return fail(TANB_INVALID_ARG, "output group %u has no channel", g);
  }
  const PcmIO pcm{in, in_step, in_gain, group, ngroups, out, out_step, out_gain};
  const int32_t r = process_common(v, Mem::Host, reinterpret_cast<const float* const*>(in), Mem::Host,
                                   reinterpret_cast<float* const*>(out), n, nullptr, done, &pcm);
  if (r == TANB_OK && clipped) *clipped = (v->h_clip && *v->h_clip) ? 1 : 0;
  return r;
}

int32_t tanb_convolution_process_direct(tanb_convolution* v, const float* const* ir, const float* const* in,
                                        float* const* out, size_t n, size_t* done, const int32_t* nz) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (done) *done = 0;
  if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "ProcessDirect before Init");
  if (!v->td) return fail(TANB_NOT_SUPPORTED, "ProcessDirect requires the TIME_DOMAIN method");
  if (!ir || !in || !out) return fail(TANB_INVALID_ARG, "null buffer array");
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  return td_process_direct(v, ir, in, out, n, done, nz);
}

int32_t tanb_convolution_process_finalize(tanb_convolution* v) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (!v->initialized) return TANB_OK;
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  return run_pending_finalize(v);
}

int32_t tanb_convolution_get_next_free_channel(tanb_convolution* v, uint32_t* idx, const uint32_t* flags) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "not initialized");
  if (!idx) return fail(TANB_INVALID_ARG, "pChannelIndex == NULL");
  *idx = 0xFFFFFFFFu;
  if (!flags) return TANB_NOT_FOUND;
  for (int c = 0; c < v->C; ++c) {
    if ((flags[c] & kStopInput) && v->tail_left[c] <= 0) {
      *idx = (uint32_t)c;
      return TANB_OK;
    }
  }
  return TANB_NOT_FOUND;
}

int32_t tanb_convolution_synchronize(tanb_convolution* v) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (!v->initialized) return TANB_OK;
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  if (v->nu_eng) return tanb_engine_synchronize(v->nu_eng);
  TANB_CUDA(cudaStreamSynchronize(v->stream));
  if (v->h_err && *v->h_err != tanb::kErrNone) return fail(TANB_FAIL, "device wait timed out (error %d)", *v->h_err);
  return TANB_OK;
}

void* tanb_convolution_stream(tanb_convolution* v) {
  if (v && v->nu_eng) return tanb_engine_stream(v->nu_eng);
  return v ? (void*)v->stream : nullptr;
}

int32_t tanb_convolution_tiling(tanb_convolution* v, int32_t index, int32_t out[3]) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (index >= tanb::mac_tiling_count()) return fail(TANB_OUT_OF_RANGE, "tiling index %d out of range", index);
  if (index >= 0) v->tiling = tanb::mac_tiling(index);
  if (out) {
    out[0] = v->tiling.ux;
    out[1] = v->tiling.sy;
    out[2] = v->tiling.depth;
  }
  return TANB_OK;
}

int32_t tanb_convolution_set_wait_limit(tanb_convolution* v, int32_t polls) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  if (polls < 0) polls = tanb::kBulkWaitLimit;
  v->ds.wait_limit = std::min(polls, tanb::kBulkWaitLimit);
  return TANB_OK;
}

int32_t tanb_convolution_profile(tanb_convolution* v, int32_t enable) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  std::lock_guard<std::mutex> lock(v->mu);
  v->profiling = enable != 0;
  return TANB_OK;
}

int32_t tanb_convolution_profile_read(tanb_convolution* v, int64_t counts[6], double ms[3]) {
  if (!v || !counts || !ms) return fail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  if (v->initialized) cudaSetDevice(v->ctx->device);
  drain_timed(v);
  for (int k = 0; k < tanb_convolution::kKinds; ++k) {
    counts[k] = v->launches[k];
    counts[3 + k] = v->timed_count[k];
    ms[k] = v->ms[k];
    v->launches[k] = 0;
    v->timed_count[k] = 0;
    v->ms[k] = 0.0;
  }
  return TANB_OK;
}

int32_t tanb_convolution_call_times(tanb_convolution* v, double us[6]) {
  if (!v || !us) return fail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  for (int k = 0; k < 6; ++k) us[k] = v->ct[k];
  return TANB_OK;
}

// ---------------------------------------------------------------------------
// Stream-state snapshot and restore (no reference counterpart): everything a
// uniformly partitioned object carries from one block to the next -- both IR
// slots' spectra, the delay line, the overlap-save history, the tail rows
// (including a pending IR's), the delay-line position, the block count (the
// tail rows alternate with its parity) and the per-channel swap and flag
// state -- so that another object with the same Init, on this GPU or on
// another, resumes the stream with the same output bit for bit: a checkpoint,
// or a session's migration between GPUs through host memory.
// ---------------------------------------------------------------------------
namespace {

struct SnapHeader {
  char magic[8];
  uint32_t method, L, B, C, P, length;
  int32_t cur;
  int64_t blocks;
};
constexpr char kSnapMagic[8] = {'T', 'A', 'N', 'B', 'S', 'N', 'P', '1'};

size_t snap_bytes(const tanb_convolution* v) {
  const size_t C = v->C, P = v->P, B = v->B;
  return sizeof(SnapHeader) + C * (4 * sizeof(int32_t) + 2) +
         (C * 2 * P * B + C * P * B + C * 3 * B) * sizeof(float2) + C * B * sizeof(float);
}

int32_t snap_check(tanb_convolution* v) {
  if (!v) return fail(TANB_INVALID_POINTER, "null convolution");
  if (!v->initialized) return fail(TANB_NOT_INITIALIZED, "snapshot before Init");
  if (v->td || v->nu_eng)
    return fail(TANB_NOT_SUPPORTED, "snapshots cover the uniformly partitioned methods");
  return TANB_OK;
}

}  // namespace

int32_t tanb_convolution_snapshot_bytes(tanb_convolution* v, uint64_t* bytes) {
  if (bytes) *bytes = 0;
  if (!v || !bytes) return fail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  const int32_t r = snap_check(v);
  if (r != TANB_OK) return r;
  *bytes = snap_bytes(v);
  return TANB_OK;
}

int32_t tanb_convolution_snapshot(tanb_convolution* v, void* buffer, uint64_t bytes) {
  if (!v || !buffer) return fail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  int32_t r = snap_check(v);
  if (r != TANB_OK) return r;
  if (bytes < snap_bytes(v)) return fail(TANB_INVALID_ARG, "snapshot buffer of %llu bytes, %zu needed",
                                         (unsigned long long)bytes, snap_bytes(v));
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  // a tail deferred by finalize mode belongs to the state: run it first
  if (run_pending_finalize(v) != TANB_OK) return TANB_FAIL;
  TANB_CUDA(cudaStreamSynchronize(v->stream));
  v->staging_busy = false;
  if (*v->h_err != tanb::kErrNone) return fail(TANB_FAIL, "device wait timed out (error %d)", *v->h_err);
  const size_t C = v->C, P = v->P, B = v->B;
  char* p = static_cast<char*>(buffer);
  SnapHeader h{};
  std::memcpy(h.magic, kSnapMagic, sizeof(h.magic));
  h.method = v->method;
  h.L = (uint32_t)v->L;
  h.B = (uint32_t)v->B;
  h.C = (uint32_t)v->C;
  h.P = (uint32_t)v->P;
  h.length = (uint32_t)v->length;
  h.cur = v->cur;
  h.blocks = v->blocks;
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  for (const std::vector<int>* a : {&v->active, &v->pending, &v->slot_new, &v->tail_left}) {
    for (size_t c = 0; c < C; ++c) {
      const int32_t x = (*a)[c];
      std::memcpy(p, &x, sizeof(x));
      p += sizeof(x);
    }
  }
  std::memcpy(p, v->available.data(), C);
  p += C;
  std::memcpy(p, v->flushed.data(), C);
  p += C;
  const size_t nh = C * 2 * P * B * sizeof(float2), nf = C * P * B * sizeof(float2), np_ = C * B * sizeof(float),
               nt = C * 3 * B * sizeof(float2);
  TANB_CUDA(cudaMemcpy(p, v->ds.H, nh, cudaMemcpyDeviceToHost));
  p += nh;
  TANB_CUDA(cudaMemcpy(p, v->ds.fdl, nf, cudaMemcpyDeviceToHost));
  p += nf;
  TANB_CUDA(cudaMemcpy(p, v->ds.prev, np_, cudaMemcpyDeviceToHost));
  p += np_;
  TANB_CUDA(cudaMemcpy(p, v->ds.tail, nt, cudaMemcpyDeviceToHost));
  return TANB_OK;
}

int32_t tanb_convolution_restore(tanb_convolution* v, const void* buffer, uint64_t bytes) {
  if (!v || !buffer) return fail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(v->mu);
  int32_t r = snap_check(v);
  if (r != TANB_OK) return r;
  if (bytes < snap_bytes(v)) return fail(TANB_INVALID_ARG, "snapshot of %llu bytes, %zu expected",
                                         (unsigned long long)bytes, snap_bytes(v));
  const char* p = static_cast<const char*>(buffer);
  SnapHeader h;
  std::memcpy(&h, p, sizeof(h));
  p += sizeof(h);
  if (std::memcmp(h.magic, kSnapMagic, sizeof(h.magic)) != 0) return fail(TANB_INVALID_ARG, "not a snapshot");
  if (h.method != v->method || h.L != (uint32_t)v->L || h.B != (uint32_t)v->B || h.C != (uint32_t)v->C ||
      h.P != (uint32_t)v->P || h.length != (uint32_t)v->length)
    return fail(TANB_INVALID_ARG, "snapshot of another configuration (method %u, L %u, B %u, C %u)", h.method, h.L,
                h.B, h.C);
  if (h.cur < 0 || h.cur >= v->P || h.blocks < 0) return fail(TANB_INVALID_ARG, "corrupt snapshot header");
  TANB_CUDA(cudaSetDevice(v->ctx->device));
  // nothing of this object's own stream may still run on the buffers
  v->finalize_due = false;
  TANB_CUDA(cudaStreamSynchronize(v->stream));
  v->staging_busy = false;
  const size_t C = v->C, P = v->P, B = v->B;
  for (std::vector<int>* a : {&v->active, &v->pending, &v->slot_new, &v->tail_left}) {
    for (size_t c = 0; c < C; ++c) {
      int32_t x;
      std::memcpy(&x, p, sizeof(x));
      p += sizeof(x);
      (*a)[c] = x;
    }
  }
  for (size_t c = 0; c < C; ++c)
    if ((v->active[c] | v->slot_new[c] | v->pending[c]) & ~1) return fail(TANB_INVALID_ARG, "corrupt snapshot state");
  std::memcpy(v->available.data(), p, C);
  p += C;
  std::memcpy(v->flushed.data(), p, C);
  p += C;
  const size_t nh = C * 2 * P * B * sizeof(float2), nf = C * P * B * sizeof(float2), np_ = C * B * sizeof(float),
               nt = C * 3 * B * sizeof(float2);
  TANB_CUDA(cudaMemcpy(v->ds.H, p, nh, cudaMemcpyHostToDevice));
  p += nh;
  TANB_CUDA(cudaMemcpy(v->ds.fdl, p, nf, cudaMemcpyHostToDevice));
  p += nf;
  TANB_CUDA(cudaMemcpy(v->ds.prev, p, np_, cudaMemcpyHostToDevice));
  p += np_;
  TANB_CUDA(cudaMemcpy(v->ds.tail, p, nt, cudaMemcpyHostToDevice));
  v->cur = h.cur;
  v->blocks = h.blocks;
  return TANB_OK;
}

int32_t tanb_convolution_info(tanb_convolution* v, int64_t out[4]) {
  if (!v || !out) return fail(TANB_INVALID_POINTER, "null argument");
  out[0] = v->nu_eng ? (int64_t)v->nu_parts[0] : v->P;  // non-uniform: the base level's partitions
  out[1] = v->B;
  out[2] = v->C;
  out[3] = (int64_t)v->dev_bytes;
  return v->initialized ? TANB_OK : TANB_NOT_INITIALIZED;
}

}  // extern "C"
