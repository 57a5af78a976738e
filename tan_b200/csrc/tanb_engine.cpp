// Batched engine behind the tanb_engine_* entry points of include/tanb.h.
//
// Many sessions (each the equivalent of one TANConvolution object: C channels,
// IR length L) share one block size and one CUDA stream. A session's IR spectra,
// delay line, overlap-save history and tail partial sums live in a
// device-memory arena sized by the caller's budget; opening a session that does
// not fit is refused with AMF_OUT_OF_MEMORY (admission by memory budget).
//
// Per audio block one CUDA graph runs a single kernel launch: the heads of every
// channel slot (reading the pinned input buffer and writing the pinned output
// buffer in place) side by side with persistent CTAs over the tail work items,
// which compute the next block's partial sums. The graph is re-instantiated
// only when the high-water marks of channel slots or work items change.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tanb.h"
#include "tanb_engine.h"
#include "tanb_host_pool.h"
#include "tanb_internal.h"

using tanb::EngChan;
using tanb::EngItem;
using tanb::EngUpd;

namespace {

int32_t efail(int32_t code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  tanb::set_last_error(buf);
  return code;
}

#define ENG_CUDA(expr)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return efail(e_ == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL,      \
                   "%s failed: %s", #expr, cudaGetErrorString(e_));                      \
  } while (0)

constexpr size_t kAlign = 256;

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// First-fit range allocator with coalescing (offsets in arbitrary units).
class RangeAlloc {
 public:
  void reset(size_t size) {
    free_.clear();
    if (size) free_[0] = size;
    size_ = size;
  }
  bool alloc(size_t n, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *off = it->first;
        size_t rest = it->second - n;
        size_t start = it->first + n;
        free_.erase(it);
        if (rest) free_[start] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t n) {
    if (!n) return;
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  // one past the highest allocated unit
  size_t high_water() const {
    if (free_.empty()) return size_;
    auto last = std::prev(free_.end());
    return (last->first + last->second == size_) ? last->first : size_;
  }

 private:
  std::map<size_t, size_t> free_;
  size_t size_ = 0;
};

struct Session {
  int id = -1;
  int C = 0, L = 0, P = 0, nitem = 0;
  size_t slot0 = 0, item0 = 0;
  size_t arena_off = 0, arena_bytes = 0;
  // IR update staged on the update stream, waiting for its event before commit
  bool staged = false;
  cudaEvent_t staged_ev = nullptr;
  int64_t blocks = 0;            // blocks processed since the session opened
  int64_t last_swap_block = -1;  // session block at which the last IR update took effect
};

}  // namespace

struct tanb_engine {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  int B = 0, log2B = 0, spec = 0, Q = 32;
  size_t budget = 0, max_channels = 0, max_items = 0;
  cudaStream_t stream = nullptr;      // audio path: head, tail, I/O copies
  cudaStream_t upd_stream = nullptr;  // IR uploads and transforms
  std::mutex upd_mu;                  // serialises IR updates (taken before mu)
  char* arena = nullptr;
  RangeAlloc arena_alloc, slot_alloc, item_alloc;
  EngChan* d_chans = nullptr;
  EngChan* h_chans = nullptr;
  EngItem* d_items = nullptr;
  EngItem* h_items = nullptr;
  float* h_in = nullptr;   // pinned; read in place by the heads
  float* h_out = nullptr;  // pinned; written in place by the heads
  long long* d_block = nullptr;     // blocks processed (device)
  unsigned int* d_done = nullptr;   // CTAs finished in the running launch
  float* h_ir = nullptr;
  float* d_ir = nullptr;
  size_t ir_cap = 0;
  EngUpd* h_upd = nullptr;
  EngUpd* d_upd = nullptr;
  float2* d_tw = nullptr;
  int tail_grid = 0;
  size_t nslots_hwm = 0, nitems_hwm = 0;
  size_t graph_slots = (size_t)-1, graph_items = (size_t)-1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t ev_out = nullptr;
  cudaEvent_t ev_audio = nullptr;  // audio-stream point an IR upload waits for
  std::map<int, Session> sessions;
  int next_id = 1;
  // accounting
  bool profiling = false;
  cudaEvent_t pa = nullptr, pb = nullptr;
  double ms_block = 0;
  int64_t n_block = 0, n_commit = 0, n_ir = 0, n_timed = 0;
};

namespace {

// Bytes per packed bin of an IR-spectrum row and of a delay-line row.
size_t spec_bytes(int spec) { return spec == tanb::kSpecFP32 ? 8 : spec == tanb::kSpecFP24 ? 6 : 4; }
size_t fdl_bytes(int spec) { return spec == tanb::kSpecFP24 ? 6 : 8; }
bool spec_scaled(int spec) { return spec == tanb::kSpecFP16 || spec == tanb::kSpecBF16; }

size_t session_bytes(const tanb_engine* e, int C, int P, int nitem) {
  const size_t B = e->B;
  size_t per = align_up(2 * (size_t)P * B * spec_bytes(e->spec));        // H
  if (spec_scaled(e->spec)) per += align_up(2 * (size_t)P * 4);          // scales
  per += align_up((size_t)P * B * fdl_bytes(e->spec));                   // fdl
  per += align_up(B * 4);                                                // prev
  per += align_up(4 * (size_t)nitem * B * 8);                            // partials
  return per * C;
}

void destroy_graph(tanb_engine* e) {
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->graph_exec = nullptr;
  e->graph = nullptr;
  e->graph_slots = e->graph_items = (size_t)-1;
}

void free_engine(tanb_engine* e) {
  if (e->upd_stream) cudaStreamSynchronize(e->upd_stream);
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (auto& kv : e->sessions)
    if (kv.second.staged_ev) cudaEventDestroy(kv.second.staged_ev);
  e->sessions.clear();
  destroy_graph(e);
  cudaFree(e->arena);
  cudaFree(e->d_chans);
  cudaFree(e->d_items);
  cudaFree(e->d_block);
  cudaFree(e->d_ir);
  cudaFree(e->d_upd);
  cudaFree(e->d_tw);
  cudaFreeHost(e->h_chans);
  cudaFreeHost(e->h_items);
  cudaFreeHost(e->h_in);
  cudaFreeHost(e->h_out);
  cudaFreeHost(e->h_ir);
  cudaFreeHost(e->h_upd);
  if (e->ev_out) cudaEventDestroy(e->ev_out);
  if (e->ev_audio) cudaEventDestroy(e->ev_audio);
  if (e->pa) cudaEventDestroy(e->pa);
  if (e->pb) cudaEventDestroy(e->pb);
  if (e->upd_stream) cudaStreamDestroy(e->upd_stream);
  if (e->stream) cudaStreamDestroy(e->stream);
}


cudaError_t upload_chans(tanb_engine* e, size_t first, size_t n) {
  if (!n) return cudaSuccess;
  return cudaMemcpyAsync(e->d_chans + first, e->h_chans + first, n * sizeof(EngChan), cudaMemcpyHostToDevice,
                         e->stream);
}

cudaError_t upload_items(tanb_engine* e, size_t first, size_t n) {
  if (!n) return cudaSuccess;
  return cudaMemcpyAsync(e->d_items + first, e->h_items + first, n * sizeof(EngItem), cudaMemcpyHostToDevice,
                         e->stream);
}

void update_hwm(tanb_engine* e) {
  e->nslots_hwm = e->slot_alloc.high_water();
  e->nitems_hwm = e->item_alloc.high_water();
}

// Commits every staged IR update whose transform has finished: the channels'
// pending flags go to the device table and the new IR's partial sums for the
// coming block are computed from the current delay line, both on the audio
// stream before this block's launch (whose heads then crossfade to the new IR).
// Caller holds mu.
cudaError_t commit_updates(tanb_engine* e) {
  for (auto& kv : e->sessions) {
    Session& s = kv.second;
    if (!s.staged) continue;
    cudaError_t q = cudaEventQuery(s.staged_ev);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return q;
    s.staged = false;
    s.last_swap_block = s.blocks;  // the head of this block crossfades to the new IR
    for (int j = 0; j < s.C; ++j) e->h_chans[s.slot0 + j].pending = 1;
    // not a copy of the mirror: process_device returns before the device has
    // run this, and the mirror advances right away
    cudaError_t r = tanb::eng_launch_mark_pending(e->d_chans, (int)s.slot0, s.C, e->stream);
    if (r != cudaSuccess) return r;
    if (s.nitem) {
      r = tanb::eng_launch_commit(e->log2B, e->spec, e->d_chans, e->d_items, (int)s.item0, s.C * s.nitem,
                                  std::min(e->tail_grid, s.C * s.nitem), e->d_block, e->stream);
      if (r != cudaSuccess) return r;
      e->n_commit += 1;
    }
  }
  return cudaSuccess;
}

// Item CTAs of the block launch: three quarters of the resident capacity, so
// that head CTAs fit beside them on every SM.
int tail_ctas(const tanb_engine* e) {
  return (int)std::min<size_t>(e->tail_grid - e->tail_grid / 4, e->nitems_hwm);
}

// Enqueues one block: the single launch over all slots and work items (in and
// out: device rows or the pinned host buffers).
cudaError_t enqueue_block(tanb_engine* e, const float* in, float* out, size_t ld) {
  return tanb::eng_launch_block(e->log2B, e->spec, e->d_chans, (int)e->nslots_hwm, e->d_items, (int)e->nitems_hwm,
                                tail_ctas(e), in, out, (int)ld, e->d_tw, tanb::EngSync{e->d_block, e->d_done},
                                e->stream);
}

cudaError_t ensure_graph(tanb_engine* e) {
  if (e->graph_exec && e->graph_slots == e->nslots_hwm && e->graph_items == e->nitems_hwm) return cudaSuccess;
  destroy_graph(e);
  cudaError_t r = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
  if (r != cudaSuccess) return r;
  cudaError_t r2 = enqueue_block(e, e->h_in, e->h_out, e->B);
  // inside stream capture a plain record only marks a capture dependency; the
  // external flag makes it an event-record node that fires on every launch
  if (r2 == cudaSuccess) r2 = cudaEventRecordWithFlags(e->ev_out, e->stream, cudaEventRecordExternal);
  r = cudaStreamEndCapture(e->stream, &e->graph);
  if (r2 != cudaSuccess) return r2;
  if (r != cudaSuccess) return r;
  r = cudaGraphInstantiate(&e->graph_exec, e->graph, 0);
  if (r != cudaSuccess) return r;
  e->graph_slots = e->nslots_hwm;
  e->graph_items = e->nitems_hwm;
  return cudaSuccess;
}

// Host mirror of what the head kernel does to the channel table.
void advance_mirror(tanb_engine* e) {
  for (auto& kv : e->sessions) {
    Session& s = kv.second;
    s.blocks += 1;
    for (int j = 0; j < s.C; ++j) {
      EngChan& ch = e->h_chans[s.slot0 + j];
      ch.cur = (ch.cur - 1 + ch.P) % ch.P;
      if (ch.pending) {
        ch.active = 1 - ch.active;
        ch.pending = 0;
      }
    }
  }
}

}  // namespace

extern "C" {

int32_t tanb_engine_create(tanb_context* ctx, uint32_t block, uint32_t spectrum, uint64_t budget_bytes,
                           uint32_t max_channels, uint32_t partitions_per_item, tanb_engine** out) {
  if (!ctx || !out) return efail(TANB_INVALID_POINTER, "null argument");
  *out = nullptr;
  if (block < 128 || block > 2048 || (block & (block - 1)))
    return efail(TANB_INVALID_ARG, "engine block must be a power of two in [128, 2048]");
  if (spectrum > tanb::kSpecFP24) return efail(TANB_INVALID_ARG, "unknown spectrum type %u", spectrum);
  if (max_channels == 0) return efail(TANB_INVALID_ARG, "max_channels == 0");
  if (partitions_per_item == 0) partitions_per_item = 32;
  tanb_engine* e = new tanb_engine();
  e->ctx = ctx;
  e->B = (int)block;
  while ((1 << e->log2B) < e->B) ++e->log2B;
  e->spec = (int)spectrum;
  e->Q = (int)partitions_per_item;
  e->budget = budget_bytes;
  e->max_channels = max_channels;
  e->max_items = (size_t)max_channels * 64;
  cudaError_t r = cudaSetDevice(ctx->device);
  if (r == cudaSuccess) r = tanb::eng_prepare();
  if (r == cudaSuccess) r = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (r == cudaSuccess) r = cudaStreamCreateWithFlags(&e->upd_stream, cudaStreamNonBlocking);
  const size_t io = e->max_channels * e->B;
  if (r == cudaSuccess) r = cudaMalloc(&e->arena, std::max<size_t>(budget_bytes, kAlign));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_chans, e->max_channels * sizeof(EngChan));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_items, e->max_items * sizeof(EngItem));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_block, 2 * sizeof(long long));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_upd, e->max_channels * sizeof(EngUpd));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_tw, 2 * e->B * sizeof(float2));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_chans, e->max_channels * sizeof(EngChan));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_items, e->max_items * sizeof(EngItem));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_in, io * sizeof(float));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_out, io * sizeof(float));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_upd, e->max_channels * sizeof(EngUpd));
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_audio, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreate(&e->pa);
  if (r == cudaSuccess) r = cudaEventCreate(&e->pb);
  if (r != cudaSuccess) {
    free_engine(e);
    delete e;
    cudaGetLastError();
    return efail(r == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "engine setup: %s",
                 cudaGetErrorString(r));
  }
  std::memset(e->h_chans, 0, e->max_channels * sizeof(EngChan));
  for (size_t i = 0; i < e->max_items; ++i) e->h_items[i] = EngItem{-1, 0, 0, 0};
  std::memset(e->h_in, 0, io * sizeof(float));
  std::memset(e->h_out, 0, io * sizeof(float));
  e->arena_alloc.reset(budget_bytes / kAlign);
  e->slot_alloc.reset(e->max_channels);
  e->item_alloc.reset(e->max_items);
  std::vector<float2> tw(2 * e->B);
  tanb::make_twiddles(2 * e->B, tw.data());
  r = cudaMemcpyAsync(e->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, e->stream);
  if (r == cudaSuccess) r = cudaMemsetAsync(e->d_chans, 0, e->max_channels * sizeof(EngChan), e->stream);
  if (r == cudaSuccess) r = upload_items(e, 0, e->max_items);
  if (e->d_block) e->d_done = reinterpret_cast<unsigned int*>(e->d_block + 1);
  if (r == cudaSuccess) r = cudaMemsetAsync(e->d_block, 0, 2 * sizeof(long long), e->stream);
  if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
  // tail CTAs of the block launch: as many as fit on the GPU at once (B / 4
  // threads each at up to 64 registers: 1024 threads per SM)
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int per_sm = std::max(1, std::min(32, 1024 / (e->B / 4)));
  e->tail_grid = sms * per_sm;
  if (r != cudaSuccess) {
    free_engine(e);
    delete e;
    return efail(TANB_FAIL, "engine init: %s", cudaGetErrorString(r));
  }
  *out = e;
  return TANB_OK;
}

int32_t tanb_engine_release(tanb_engine* e) {
  if (!e) return TANB_OK;
  {
    std::lock_guard<std::mutex> lock(e->mu);
    cudaSetDevice(e->ctx->device);
    free_engine(e);
  }
  delete e;
  return TANB_OK;
}

int32_t tanb_engine_open_session(tanb_engine* e, uint32_t channels, uint32_t ir_length, int32_t* session,
                                 uint32_t* first_slot) {
  if (!e || !session) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  if (channels == 0 || ir_length == 0) return efail(TANB_INVALID_ARG, "channels and IR length must be > 0");
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  Session s;
  s.C = (int)channels;
  s.L = (int)ir_length;
  s.P = (int)std::max<uint32_t>(1, (ir_length + e->B - 1) / e->B);
  // work items cover partitions [2, P); the head does partitions 0 and 1
  s.nitem = s.P > 2 ? (s.P - 2 + e->Q - 1) / e->Q : 0;
  s.arena_bytes = session_bytes(e, s.C, s.P, s.nitem);
  if (!e->arena_alloc.alloc(s.arena_bytes / kAlign, &s.arena_off))
    return efail(TANB_OUT_OF_MEMORY, "session of %u channels x %u taps needs %zu bytes; device budget exhausted",
                 channels, ir_length, s.arena_bytes);
  if (!e->slot_alloc.alloc(s.C, &s.slot0)) {
    e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
    return efail(TANB_OUT_OF_MEMORY, "no %u free channel slots", channels);
  }
  const size_t nit_total = (size_t)s.C * s.nitem;
  if (nit_total && !e->item_alloc.alloc(nit_total, &s.item0)) {
    e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
    e->slot_alloc.release(s.slot0, s.C);
    return efail(TANB_OUT_OF_MEMORY, "work-item table full");
  }
  ENG_CUDA(cudaStreamSynchronize(e->stream));  // pinned mirrors are rewritten below
  char* base = e->arena + s.arena_off * kAlign;
  ENG_CUDA(cudaMemsetAsync(base, 0, s.arena_bytes, e->stream));
  const size_t B = e->B;
  for (int j = 0; j < s.C; ++j) {
    EngChan ch{};
    ch.H = base;
    base += align_up(2 * (size_t)s.P * B * spec_bytes(e->spec));
    if (spec_scaled(e->spec)) {
      ch.scale = reinterpret_cast<float*>(base);
      base += align_up(2 * (size_t)s.P * 4);
    }
    ch.fdl = reinterpret_cast<float2*>(base);
    base += align_up((size_t)s.P * B * fdl_bytes(e->spec));
    ch.prev = reinterpret_cast<float*>(base);
    base += align_up(B * 4);
    ch.part = reinterpret_cast<float2*>(base);
    base += align_up(4 * (size_t)s.nitem * B * 8);
    ch.P = s.P;
    ch.nitem = s.nitem;
    ch.cur = 0;
    ch.active = 0;
    ch.pending = 0;
    ch.run = 1;
    e->h_chans[s.slot0 + j] = ch;
    for (int r = 0; r < s.nitem; ++r) {
      const int i0 = 2 + r * e->Q;
      e->h_items[s.item0 + (size_t)j * s.nitem + r] = EngItem{(int)(s.slot0 + j), i0, std::min(s.P, i0 + e->Q), r};
    }
  }
  ENG_CUDA(upload_chans(e, s.slot0, s.C));
  ENG_CUDA(upload_items(e, s.item0, nit_total));
  // the copies read the pinned mirrors, which the next block advances
  ENG_CUDA(cudaStreamSynchronize(e->stream));
  ENG_CUDA(cudaEventCreateWithFlags(&s.staged_ev, cudaEventDisableTiming));
  s.id = e->next_id++;
  e->sessions[s.id] = s;
  update_hwm(e);
  *session = s.id;
  if (first_slot) *first_slot = (uint32_t)s.slot0;
  return TANB_OK;
}

int32_t tanb_engine_close_session(tanb_engine* e, int32_t session) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> ulock(e->upd_mu);  // no IR upload may still write this session's memory
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->sessions.find(session);
  if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  ENG_CUDA(cudaStreamSynchronize(e->upd_stream));
  ENG_CUDA(cudaStreamSynchronize(e->stream));
  const Session s = it->second;
  if (s.staged_ev) cudaEventDestroy(s.staged_ev);
  for (int j = 0; j < s.C; ++j) e->h_chans[s.slot0 + j] = EngChan{};
  const size_t nit_total = (size_t)s.C * s.nitem;
  for (size_t i = 0; i < nit_total; ++i) e->h_items[s.item0 + i] = EngItem{-1, 0, 0, 0};
  ENG_CUDA(upload_chans(e, s.slot0, s.C));
  ENG_CUDA(upload_items(e, s.item0, nit_total));
  ENG_CUDA(cudaStreamSynchronize(e->stream));  // the copies read the pinned mirrors
  e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
  e->slot_alloc.release(s.slot0, s.C);
  e->item_alloc.release(s.item0, nit_total);
  e->sessions.erase(it);
  update_hwm(e);
  return TANB_OK;
}

static int32_t engine_update(tanb_engine* e, int32_t session, const float* const* ir, size_t n, bool device,
                             uint32_t op) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  if (!ir) return efail(TANB_INVALID_ARG, "ppBuffer == NULL");
  std::lock_guard<std::mutex> ulock(e->upd_mu);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  // the previous upload's copies read the pinned staging rewritten below
  ENG_CUDA(cudaStreamSynchronize(e->upd_stream));
  Session s;
  {
    // read the session and choose the idle IR slots under the main lock: the
    // audio path flips slots only under this lock, so the choice is consistent
    std::lock_guard<std::mutex> lock(e->mu);
    auto it = e->sessions.find(session);
    if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
    s = it->second;
    if (n > (size_t)s.L) return efail(TANB_INVALID_ARG, "IR length %zu exceeds the session's %d", n, s.L);
    for (int j = 0; j < s.C; ++j) {
      if (!ir[j] && n) return efail(TANB_INVALID_ARG, "ppBuffer[%d] == NULL", j);
      e->h_upd[j] = EngUpd{(int)(s.slot0 + j), 1 - e->h_chans[s.slot0 + j].active, nullptr, (int64_t)n};
    }
    it->second.staged = false;  // a newer upload supersedes one not yet committed
    // The mirror (and so the idle-slot choice) already reflects every block
    // enqueued on the audio stream; blocks still running there may read the
    // chosen slot (a crossfade from it), so the transform waits for them.
    ENG_CUDA(cudaEventRecord(e->ev_audio, e->stream));
    ENG_CUDA(cudaStreamWaitEvent(e->upd_stream, e->ev_audio, 0));
  }
  const size_t PB = (size_t)s.P * e->B;
  const size_t need = PB * s.C;
  if (need > e->ir_cap) {
    cudaFree(e->d_ir);
    cudaFreeHost(e->h_ir);
    e->d_ir = nullptr;
    e->h_ir = nullptr;
    e->ir_cap = 0;
    ENG_CUDA(cudaMalloc(&e->d_ir, need * sizeof(float)));
    ENG_CUDA(cudaMallocHost(&e->h_ir, need * sizeof(float)));
    e->ir_cap = need;
  }
  if (device) {
    // the transform reads the caller's rows in place
    for (int j = 0; j < s.C; ++j) e->h_upd[j].src = ir[j];
  } else if (n) {
    // compact staging (row stride n) copied on the host pool, one transfer
    auto copy_row = [&](int j) { tanb::copy_for_device(e->h_ir + (size_t)j * n, ir[j], n * sizeof(float)); };
    if ((size_t)s.C * n * sizeof(float) >= (1u << 20))
      tanb::host_parallel_for(s.C, copy_row);
    else
      for (int j = 0; j < s.C; ++j) copy_row(j);
    ENG_CUDA(cudaMemcpyAsync(e->d_ir, e->h_ir, (size_t)s.C * n * sizeof(float), cudaMemcpyHostToDevice,
                             e->upd_stream));
    for (int j = 0; j < s.C; ++j) e->h_upd[j].src = e->d_ir + (size_t)j * n;
  }
  ENG_CUDA(cudaMemcpyAsync(e->d_upd, e->h_upd, s.C * sizeof(EngUpd), cudaMemcpyHostToDevice, e->upd_stream));
  ENG_CUDA(tanb::eng_launch_ir(e->log2B, e->spec, e->d_chans, e->d_upd, s.C, s.P, e->d_tw, e->upd_stream));
  ENG_CUDA(cudaEventRecord(s.staged_ev, e->upd_stream));
  // BLOCK_UNTIL_READY: the new IR is ready for the next block when this returns
  if (op & TANB_OPERATION_FLAG_BLOCK_UNTIL_READY) ENG_CUDA(cudaEventSynchronize(s.staged_ev));
  {
    std::lock_guard<std::mutex> lock(e->mu);
    auto it = e->sessions.find(session);
    if (it != e->sessions.end()) it->second.staged = true;
    e->n_ir += 1;
  }
  return TANB_OK;
}

int32_t tanb_engine_update_response_td(tanb_engine* e, int32_t session, const float* const* ir, size_t n,
                                       uint32_t operationFlags) {
  return engine_update(e, session, ir, n, false, operationFlags);
}

int32_t tanb_engine_update_response_td_device(tanb_engine* e, int32_t session, const float* const* ir,
                                              size_t n, uint32_t operationFlags) {
  return engine_update(e, session, ir, n, true, operationFlags);
}

int32_t tanb_engine_io(tanb_engine* e, float** in, float** out) {
  if (!e || !in || !out) return efail(TANB_INVALID_POINTER, "null argument");
  *in = e->h_in;
  *out = e->h_out;
  return TANB_OK;
}

int32_t tanb_engine_write_input(tanb_engine* e, uint32_t first_slot, const float* src, uint32_t count, size_t ld) {
  if (!e || (!src && count)) return efail(TANB_INVALID_POINTER, "null argument");
  if ((size_t)first_slot + count > e->max_channels) return efail(TANB_INVALID_ARG, "slots out of range");
  if (count && ld < (size_t)e->B) return efail(TANB_INVALID_ARG, "ld %zu < block %d", ld, e->B);
  const size_t B = e->B;
  constexpr uint32_t kRowsPerTask = 64;
  const uint32_t tasks = (count + kRowsPerTask - 1) / kRowsPerTask;
  auto copy = [&](int t) {
    const uint32_t r0 = (uint32_t)t * kRowsPerTask, r1 = std::min(count, r0 + kRowsPerTask);
    // streaming stores: the heads read these rows over the bus, and rows
    // left dirty in the CPU caches are read back far more slowly
    for (uint32_t r = r0; r < r1; ++r)
      tanb::copy_rows_for_device(e->h_in + (size_t)(first_slot + r) * B, src + (size_t)r * ld, B * sizeof(float));
    tanb::copy_for_device_fence();
  };
  if ((size_t)count * B * sizeof(float) >= (1u << 20))
    tanb::host_parallel_for((int)tasks, copy);
  else
    for (uint32_t t = 0; t < tasks; ++t) copy((int)t);
  return TANB_OK;
}

int32_t tanb_engine_process(tanb_engine* e) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> lock(e->mu);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  if (e->sessions.empty()) return efail(TANB_WRONG_STATE, "no open sessions");
  ENG_CUDA(commit_updates(e));
  ENG_CUDA(ensure_graph(e));
  ENG_CUDA(cudaGraphLaunch(e->graph_exec, e->stream));
  ENG_CUDA(cudaEventSynchronize(e->ev_out));
  e->n_block += 1;
  advance_mirror(e);
  return TANB_OK;
}

int32_t tanb_engine_process_device(tanb_engine* e, const float* in, float* out, uint32_t ld) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> lock(e->mu);
  if (!out) return efail(TANB_INVALID_ARG, "null output");
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  if (e->sessions.empty()) return efail(TANB_WRONG_STATE, "no open sessions");
  if (ld == 0) ld = e->B;
  ENG_CUDA(commit_updates(e));
  if (e->profiling) ENG_CUDA(cudaEventRecord(e->pa, e->stream));
  ENG_CUDA(enqueue_block(e, in, out, ld));
  if (e->profiling) {
    ENG_CUDA(cudaEventRecord(e->pb, e->stream));
    ENG_CUDA(cudaEventSynchronize(e->pb));
    float a = 0;
    cudaEventElapsedTime(&a, e->pa, e->pb);
    e->ms_block += a;
    e->n_timed += 1;
  }
  e->n_block += 1;
  advance_mirror(e);
  return TANB_OK;
}

int32_t tanb_engine_synchronize(tanb_engine* e) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> lock(e->mu);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  ENG_CUDA(cudaStreamSynchronize(e->upd_stream));
  ENG_CUDA(cudaStreamSynchronize(e->stream));
  return TANB_OK;
}

void* tanb_engine_stream(tanb_engine* e) { return e ? (void*)e->stream : nullptr; }

int32_t tanb_engine_info(tanb_engine* e, int64_t out[8]) {
  if (!e || !out) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  int64_t chans = 0, bytes = 0, block_bytes = 0;
  const int64_t B = e->B, sb = (int64_t)spec_bytes(e->spec), xb = (int64_t)fdl_bytes(e->spec);
  for (auto& kv : e->sessions) {
    const Session& s = kv.second;
    chans += s.C;
    bytes += (int64_t)s.arena_bytes;
    // algorithmic bytes of one block launch per channel: tail items stream
    // partitions [2, P) of IR spectrum and delay line and write their partial
    // rows; the head reads input, history, the partial rows, partitions 0 and
    // 1 of the spectrum and X_{k-1}, and writes output, history and X_k
    const int64_t tail = (s.P > 2 ? (int64_t)(s.P - 2) * B * (sb + xb) : 0) + (int64_t)s.nitem * B * 8;
    const int64_t head = 4 * B * 4 + (int64_t)s.nitem * B * 8 + (s.P > 1 ? 2 * B * sb + B * xb : B * sb) + B * xb;
    block_bytes += (int64_t)s.C * (tail + head);
  }
  out[0] = (int64_t)e->sessions.size();
  out[1] = chans;
  out[2] = (int64_t)e->nslots_hwm;
  out[3] = (int64_t)e->nitems_hwm;
  out[4] = bytes;
  out[5] = (int64_t)e->budget;
  out[6] = block_bytes;
  out[7] = e->tail_grid;
  return TANB_OK;
}

int32_t tanb_engine_session_state(tanb_engine* e, int32_t session, int64_t out[3]) {
  if (!e || !out) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->sessions.find(session);
  if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
  out[0] = it->second.blocks;
  out[1] = it->second.last_swap_block;
  out[2] = it->second.staged ? 1 : 0;
  return TANB_OK;
}

int32_t tanb_engine_profile(tanb_engine* e, int32_t enable) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> lock(e->mu);
  e->profiling = enable != 0;
  return TANB_OK;
}

int32_t tanb_engine_profile_read(tanb_engine* e, int64_t counts[4], double ms[2]) {
  if (!e || !counts || !ms) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  counts[0] = e->n_block;
  counts[1] = e->n_commit;
  counts[2] = e->n_ir;
  counts[3] = e->n_timed;
  ms[0] = e->ms_block;
  ms[1] = 0.0;
  e->n_block = e->n_commit = e->n_ir = e->n_timed = 0;
  e->ms_block = 0;
  return TANB_OK;
}

}  // extern "C"
