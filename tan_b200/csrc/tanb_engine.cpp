// Batched engine behind the tanb_engine_* entry points of include/tanb.h.
//
// Many sessions (each the equivalent of one TANConvolution object: C channels,
// IR length L) share one block size and one CUDA stream. A session's IR spectra,
// delay line, overlap-save history and tail partial sums live in a
// device-memory arena sized by the caller's budget; opening a session that does
// not fit is refused with AMF_OUT_OF_MEMORY (admission by memory budget).
//
// A session is uniformly partitioned (partitions of the block size) or
// non-uniformly partitioned (a base level at the block size and levels of
// growing block sizes further along the IR, tanb_engine_open_session_nu).
//
// Per audio block one CUDA graph runs: a single block launch with the heads of
// every channel slot (reading the input rows and writing the output rows in
// place) side by side with persistent CTAs over the tail work items (the next
// block's partial sums, and one bin slice of every non-uniform level's tail),
// and, at the blocks where a level size completes, the level heads of that size
// in a kernel beside it (a parallel branch of the same graph). The graph of each
// set of due level sizes is instantiated once and re-instantiated only when the
// high-water marks of channel slots, work items or level records change.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tanb.h"
#include "tanb_engine.h"
#include "tanb_engine_host.h"
#include "tanb_host_pool.h"
#include "tanb_internal.h"

using tanb::EngChan;
using tanb::EngItem;
using tanb::EngLevel;
using tanb::EngLvlUpd;
using tanb::EngNu;
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

size_t pow2_at_least(size_t x) {
  size_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

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
  // extends the range to [0, size) (size >= the current size)
  void grow(size_t size) {
    if (size > size_) release(size_, size - size_);
    size_ = std::max(size_, size);
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

// Shape of one level above the base level of a non-uniform session.
struct LevelSpec {
  int log2N = 0, K = 0, Kr = 0, ngroup = 0, R = 0;
  int q = 0;    // partitions per work item (group)
  long long off = 0;
  int nfl = 0;  // level blocks whose output an IR swap recomputes (at most)
};

struct Session {
  int id = -1;
  int C = 0, L = 0, P = 0, nitem = 0;  // P, nitem: the (base) level at the engine block
  int items_per_chan = 0;              // base items + level items per channel
  size_t slot0 = 0, item0 = 0;
  size_t arena_off = 0, arena_bytes = 0;
  std::vector<LevelSpec> lv;           // levels above the base level (empty: uniform)
  std::vector<size_t> lv_first;        // per level: its C consecutive records in the size class's table
  int rin = 0;                         // input history length (non-uniform)
  // IR update staged on the update stream, waiting for its event before commit
  bool staged = false;
  cudaEvent_t staged_ev = nullptr;
  std::vector<uint8_t> staged_mask;    // channels the staged update replaces
  int64_t blocks = 0;            // blocks processed since the session opened
  int64_t last_swap_block = -1;  // session block at which the last IR update took effect
  // per channel: the device ranges a flush clears (delay lines, history,
  // partial sums, level rings)
  std::vector<std::vector<std::pair<char*, size_t>>> zero;
};

}  // namespace

struct tanb_engine {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  int B = 0, log2B = 0, spec = 0, Q = 32;
  size_t budget = 0, max_channels = 0, max_items = 0;
  cudaStream_t stream = nullptr;      // audio path: blocks, commits
  std::vector<cudaStream_t> lstreams;  // level heads beside the block launch, one stream per size class
  cudaStream_t upd_stream = nullptr;  // IR uploads and transforms
  std::mutex upd_mu;                  // serialises IR updates (taken before mu)
  char* arena = nullptr;
  RangeAlloc arena_alloc, slot_alloc, item_alloc;
  EngChan* d_chans = nullptr;
  EngChan* h_chans = nullptr;
  EngItem* d_items = nullptr;
  EngItem* h_items = nullptr;
  // level records: size class c (level block 2^(log2B + 1 + c)) at [c * max_channels, (c + 1) * max_channels)
  int nclass = 0;
  EngLevel* d_levels = nullptr;
  EngLevel* h_levels = nullptr;
  std::vector<RangeAlloc> lvl_alloc;
  std::vector<size_t> lvl_hwm;
  std::vector<float2*> d_tw_lv;       // twiddles of each size class (2N entries)
  float* h_in = nullptr;   // pinned; read in place by the heads
  float* h_out = nullptr;  // pinned; written in place by the heads
  long long* d_block = nullptr;     // blocks processed (device)
  unsigned int* d_done = nullptr;   // CTAs finished in the running block
  long long k_host = 0;             // blocks enqueued (the device counter after they ran)
  float* h_ir = nullptr;
  float* d_ir = nullptr;
  size_t ir_cap = 0;
  EngUpd* h_upd = nullptr;
  EngUpd* d_upd = nullptr;
  EngLvlUpd* h_lupd = nullptr;
  EngLvlUpd* d_lupd = nullptr;
  float2* d_tw = nullptr;
  int tail_grid = 0;
  int sms = 148;  // SMs of the device
  size_t nslots_hwm = 0, nitems_hwm = 0;
  // graphs of the host-buffer block, one per set of due level size classes,
  // each valid for the high-water marks in its key; executable graphs
  // replaced on the audio path are retired, not destroyed, there (destroying
  // one can wait for the device) and destroyed by synchronize and release
  struct BlockGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<size_t> key;
  };
  std::map<unsigned, BlockGraph> graphs;
  std::vector<cudaGraphExec_t> retired;
  cudaEvent_t ev_out = nullptr;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_joins;  // one per level size class
  cudaEvent_t ev_audio = nullptr;  // audio-stream point an IR upload waits for
  // Pinned staging of the table uploads of session opens and closes: they copy
  // from here rather than from the live mirrors (which the audio path keeps
  // advancing), so that an open or a close never waits for the audio stream.
  char* h_stage = nullptr;
  size_t stage_cap = 0, stage_used = 0;
  cudaEvent_t ev_stage = nullptr;   // behind the last staged upload
  cudaEvent_t ev_upd_done = nullptr;  // update-stream point a close orders the audio stream after
  std::map<int, Session> sessions;
  int next_id = 1;
  // accounting
  bool profiling = false;
  cudaEvent_t pa = nullptr, pb = nullptr;
  double ms_block = 0;
  int64_t n_block = 0, n_commit = 0, n_ir = 0, n_timed = 0;
  // host microseconds of the last tanb_engine_process (tanb_engine_block_times)
  double bt_lock = 0, bt_commit = 0, bt_build = 0, bt_launch = 0, bt_wait = 0, bt_total = 0, bt_max = 0;
  int64_t n_graph_builds = 0;
};

namespace {

using Clock = std::chrono::steady_clock;
double us_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
}

// Bytes per packed bin of an IR-spectrum row and of a delay-line row.
size_t spec_bytes(int spec) { return spec == tanb::kSpecFP32 ? 8 : spec == tanb::kSpecFP24 ? 6 : 4; }
size_t fdl_bytes(int spec) { return spec == tanb::kSpecFP24 ? 6 : 8; }
bool spec_scaled(int spec) { return spec == tanb::kSpecFP16 || spec == tanb::kSpecBF16; }

size_t chan_bytes(const tanb_engine* e, int P, int nitem, const std::vector<LevelSpec>& lv, int rin) {
  const size_t B = e->B;
  size_t per = align_up(2 * (size_t)P * B * spec_bytes(e->spec));        // H
  if (spec_scaled(e->spec)) per += align_up(2 * (size_t)P * 4);          // scales
  per += align_up((size_t)P * B * fdl_bytes(e->spec));                   // fdl
  per += align_up(B * 4);                                                // prev
  per += align_up(4 * (size_t)nitem * B * 8);                            // partials
  if (!lv.empty()) {
    per += align_up(sizeof(EngNu)) + align_up((size_t)rin * 4);
    for (const LevelSpec& l : lv) {
      const size_t N = (size_t)1 << l.log2N;
      per += align_up(2 * (size_t)l.K * N * spec_bytes(e->spec));
      if (spec_scaled(e->spec)) per += align_up(2 * (size_t)l.K * 4);
      per += align_up((size_t)l.Kr * N * fdl_bytes(e->spec));
      per += align_up(2 * (size_t)l.ngroup * N * 8);
      per += align_up(2 * (size_t)l.R * 4);
    }
  }
  return per;
}

int level_class(const tanb_engine* e, int log2N) { return log2N - e->log2B - 1; }

constexpr size_t kMaxRetiredGraphs = 64;

void destroy_retired(tanb_engine* e) {
  for (cudaGraphExec_t g : e->retired) cudaGraphExecDestroy(g);
  e->retired.clear();
}

void destroy_graphs(tanb_engine* e) {
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second.exec);
  e->graphs.clear();
  destroy_retired(e);
}

void free_engine(tanb_engine* e) {
  if (e->upd_stream) cudaStreamSynchronize(e->upd_stream);
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (cudaStream_t ls : e->lstreams)
    if (ls) cudaStreamSynchronize(ls);
  for (auto& kv : e->sessions)
    if (kv.second.staged_ev) cudaEventDestroy(kv.second.staged_ev);
  e->sessions.clear();
  destroy_graphs(e);
  cudaFree(e->arena);
  cudaFree(e->d_chans);
  cudaFree(e->d_items);
  cudaFree(e->d_levels);
  cudaFree(e->d_block);
  cudaFree(e->d_ir);
  cudaFree(e->d_upd);
  cudaFree(e->d_lupd);
  cudaFree(e->d_tw);
  for (float2* t : e->d_tw_lv) cudaFree(t);
  cudaFreeHost(e->h_chans);
  cudaFreeHost(e->h_items);
  cudaFreeHost(e->h_levels);
  cudaFreeHost(e->h_in);
  cudaFreeHost(e->h_out);
  cudaFreeHost(e->h_ir);
  cudaFreeHost(e->h_upd);
  cudaFreeHost(e->h_lupd);
  cudaFreeHost(e->h_stage);
  if (e->ev_stage) cudaEventDestroy(e->ev_stage);
  if (e->ev_upd_done) cudaEventDestroy(e->ev_upd_done);
  if (e->ev_out) cudaEventDestroy(e->ev_out);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  for (cudaEvent_t ev : e->ev_joins)
    if (ev) cudaEventDestroy(ev);
  if (e->ev_audio) cudaEventDestroy(e->ev_audio);
  if (e->pa) cudaEventDestroy(e->pa);
  if (e->pb) cudaEventDestroy(e->pb);
  if (e->upd_stream) cudaStreamDestroy(e->upd_stream);
  for (cudaStream_t ls : e->lstreams)
    if (ls) cudaStreamDestroy(ls);
  if (e->stream) cudaStreamDestroy(e->stream);
}

cudaError_t upload_items(tanb_engine* e, size_t first, size_t n) {
  if (!n) return cudaSuccess;
  return cudaMemcpyAsync(e->d_items + first, e->h_items + first, n * sizeof(EngItem), cudaMemcpyHostToDevice,
                         e->stream);
}

cudaError_t upload_levels(tanb_engine* e, size_t first, size_t n) {
  if (!n) return cudaSuccess;
  return cudaMemcpyAsync(e->d_levels + first, e->h_levels + first, n * sizeof(EngLevel), cudaMemcpyHostToDevice,
                         e->stream);
}

// Staged uploads (see tanb_engine::h_stage): begin_stage waits for the
// previous staged uploads to have run (long done in practice) and makes room
// for `bytes`; stage_copy queues one copy on the audio stream; end_stage marks
// the point the next begin_stage waits for.
cudaError_t begin_stage(tanb_engine* e, size_t bytes) {
  cudaError_t r = cudaEventSynchronize(e->ev_stage);
  if (r != cudaSuccess) return r;
  if (bytes > e->stage_cap) {
    cudaFreeHost(e->h_stage);
    e->h_stage = nullptr;
    e->stage_cap = 0;
    if ((r = cudaMallocHost(&e->h_stage, bytes)) != cudaSuccess) return r;
    e->stage_cap = bytes;
  }
  e->stage_used = 0;
  return cudaSuccess;
}

cudaError_t stage_copy(tanb_engine* e, void* dev, const void* host, size_t bytes) {
  if (!bytes) return cudaSuccess;
  if (e->stage_used + bytes > e->stage_cap) return cudaErrorInvalidValue;
  char* src = e->h_stage + e->stage_used;
  std::memcpy(src, host, bytes);
  e->stage_used += (bytes + 15) & ~size_t(15);
  return cudaMemcpyAsync(dev, src, bytes, cudaMemcpyHostToDevice, e->stream);
}

cudaError_t end_stage(tanb_engine* e) { return cudaEventRecord(e->ev_stage, e->stream); }

void update_hwm(tanb_engine* e) {
  e->nslots_hwm = e->slot_alloc.high_water();
  e->nitems_hwm = e->item_alloc.high_water();
  for (int c = 0; c < e->nclass; ++c) e->lvl_hwm[c] = e->lvl_alloc[c].high_water();
}

// Commits every staged IR update whose transform has finished: the channels'
// pending flags go to the device table, the new IR's partial sums for the
// coming block are computed from the current delay line and, for non-uniform
// sessions, the levels' partial sums of the level blocks still to come and the
// output of level blocks still to be played, all on the audio stream before
// this block's launch (whose heads then crossfade to the new IR).
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
    // runs of updated channels; not a copy of the mirror: process returns
    // before the device has run this, and the mirror advances right away
    for (int j = 0; j < s.C;) {
      if (!s.staged_mask[j]) {
        ++j;
        continue;
      }
      int j1 = j;
      while (j1 < s.C && s.staged_mask[j1]) e->h_chans[s.slot0 + j1++].pending = 1;
      cudaError_t r = tanb::eng_launch_mark_pending(e->d_chans, (int)s.slot0 + j, j1 - j, e->stream);
      if (r != cudaSuccess) return r;
      j = j1;
    }
    const int nit = s.C * s.items_per_chan;
    const int grid = std::max(1, std::min(e->tail_grid, nit));
    cudaError_t r = cudaSuccess;
    if (s.nitem)
      r = tanb::eng_launch_commit(e->log2B, e->spec, e->d_chans, e->d_items, (int)s.item0, nit, grid, e->d_block,
                                  e->stream);
    if (r == cudaSuccess && nit > 2 * s.C * s.nitem) {
      int slices = 1;  // bin slices of the largest level with work items
      for (const LevelSpec& l : s.lv)
        if (l.ngroup) slices = std::max(slices, 1 << (l.log2N - e->log2B));
      const long long pairs = (long long)nit * slices;
      r = tanb::eng_launch_level_commit_items(e->log2B, e->spec, e->d_chans, e->d_levels, e->d_items, (int)s.item0,
                                              nit, slices, (int)std::min<long long>(e->tail_grid, pairs), e->d_block,
                                              e->stream);
    }
    for (size_t l = 0; l < s.lv.size() && r == cudaSuccess; ++l) {
      const int c = level_class(e, s.lv[l].log2N);
      r = tanb::eng_launch_level_commit_out(e->log2B, s.lv[l].log2N, e->spec, e->d_chans,
                                            e->d_levels + (size_t)c * e->max_channels, (int)s.lv_first[l], s.C,
                                            s.lv[l].nfl, e->d_tw_lv[c], e->d_block, e->stream);
    }
    if (r != cudaSuccess) return r;
    e->n_commit += 1;
  }
  return cudaSuccess;
}

// Item CTAs of the block launch: three quarters of the resident capacity, so
// that head CTAs fit beside them on every SM.
int tail_ctas(const tanb_engine* e) {
  return (int)std::min<size_t>(e->tail_grid - e->tail_grid / 4, e->nitems_hwm);
}

// Level size classes due at block k (bit c: class c has records and its
// block completes with base block k).
unsigned due_mask(const tanb_engine* e, long long k) {
  unsigned m = 0;
  for (int c = 0; c < e->nclass; ++c) {
    const long long p = 2LL << c;  // N / B
    if (e->lvl_hwm[c] && ((k + 1) % p) == 0) m |= 1u << c;
  }
  return m;
}

// Enqueues one block: the block launch over all slots and work items, and the
// heads of each due level class on that class's stream beside it (forked from
// and joined back into the audio stream, so that a captured graph holds them
// as parallel branches).
cudaError_t enqueue_block(tanb_engine* e, const tanb::EngRows& rows, unsigned due) {
  const int tc = tail_ctas(e);
  unsigned total = tanb::eng_block_ctas((int)e->nslots_hwm, tc);
  for (int c = 0; c < e->nclass; ++c)
    if (due >> c & 1u) total += (unsigned)e->lvl_hwm[c];
  const tanb::EngSync sync{e->d_block, e->d_done};
  cudaError_t r;
  if (due) {
    if ((r = cudaEventRecord(e->ev_fork, e->stream)) != cudaSuccess) return r;
    for (int c = 0; c < e->nclass; ++c)
      if ((due >> c & 1u) && (r = cudaStreamWaitEvent(e->lstreams[c], e->ev_fork, 0)) != cudaSuccess) return r;
  }
  // at most two heads per SM: their transforms read the twiddles from shared
  // memory (the latency of the heads bounds such a launch); more heads share
  // them in L1 (the item CTAs' streaming bounds it)
  const bool tw_stage = e->nslots_hwm <= 2 * (size_t)e->sms;
  r = tanb::eng_launch_block(e->log2B, e->spec, e->d_chans, (int)e->nslots_hwm, e->d_items, (int)e->nitems_hwm, tc,
                             e->d_levels, rows, e->d_tw, tw_stage, sync, total, e->stream);
  if (r != cudaSuccess || !due) return r;
  for (int c = 0; c < e->nclass; ++c) {
    if (!(due >> c & 1u)) continue;
    r = tanb::eng_launch_level_heads(e->log2B, e->log2B + 1 + c, e->spec, e->d_chans, (int)e->nslots_hwm,
                                     e->d_levels + (size_t)c * e->max_channels, (int)e->lvl_hwm[c], rows,
                                     e->d_tw_lv[c], sync, total, e->lstreams[c]);
    if (r != cudaSuccess) return r;
    if ((r = cudaEventRecord(e->ev_joins[c], e->lstreams[c])) != cudaSuccess) return r;
    if ((r = cudaStreamWaitEvent(e->stream, e->ev_joins[c], 0)) != cudaSuccess) return r;
  }
  return cudaSuccess;
}

std::vector<size_t> graph_key(const tanb_engine* e) {
  std::vector<size_t> k{e->nslots_hwm, e->nitems_hwm, e->max_items};
  k.insert(k.end(), e->lvl_hwm.begin(), e->lvl_hwm.end());
  return k;
}

// The block graph for `due`, captured anew when the high-water marks changed
// since it was built: the cached executable is updated in place when the new
// capture has its topology (grid sizes and parameters differ), else a new one
// is instantiated and the old one retired.
cudaError_t ensure_graph(tanb_engine* e, unsigned due, cudaGraphExec_t* out) {
  const std::vector<size_t> key = graph_key(e);
  auto it = e->graphs.find(due);
  if (it != e->graphs.end() && it->second.key == key) {
    *out = it->second.exec;
    return cudaSuccess;
  }
  const Clock::time_point t0 = Clock::now();
  cudaGraph_t g = nullptr;
  cudaError_t r = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
  if (r != cudaSuccess) return r;
  tanb::EngRows rows;
  rows.in_base = e->h_in;
  rows.out_base = e->h_out;
  rows.ld = e->B;
  cudaError_t r2 = enqueue_block(e, rows, due);
  // inside stream capture a plain record only marks a capture dependency; the
  // external flag makes it an event-record node that fires on every launch
  if (r2 == cudaSuccess) r2 = cudaEventRecordWithFlags(e->ev_out, e->stream, cudaEventRecordExternal);
  r = cudaStreamEndCapture(e->stream, &g);
  if (r2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return r2;
  }
  if (r != cudaSuccess) return r;
  if (it != e->graphs.end()) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(it->second.exec, g, &info) == cudaSuccess) {
      cudaGraphDestroy(g);
      it->second.key = key;
      *out = it->second.exec;
      e->n_graph_builds += 1;
      e->bt_build += us_since(t0);
      return cudaSuccess;
    }
    (void)cudaGetLastError();  // a refused update leaves the executable as it was
    if (e->retired.size() >= kMaxRetiredGraphs) destroy_retired(e);
    e->retired.push_back(it->second.exec);
    e->graphs.erase(it);
  }
  cudaGraphExec_t ge = nullptr;
  r = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (r != cudaSuccess) return r;
  e->graphs[due] = tanb_engine::BlockGraph{ge, key};
  *out = ge;
  e->n_graph_builds += 1;
  e->bt_build += us_since(t0);
  return cudaSuccess;
}

// Host mirror of what the block launch does to the channel table.
void advance_mirror(tanb_engine* e) {
  e->k_host += 1;
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

// Checks a non-uniform level schedule and derives its level shapes.
int32_t make_levels(const tanb_engine* e, uint32_t ir_length, uint32_t nlevels, const uint32_t* block,
                    const uint32_t* parts, std::vector<LevelSpec>* lv, int* P0, int* rin) {
  if (nlevels == 0 || nlevels > (uint32_t)tanb::kMaxLevels + 1)
    return efail(TANB_INVALID_ARG, "a non-uniform schedule has 1 to %d levels", tanb::kMaxLevels + 1);
  if (block[0] != (uint32_t)e->B) return efail(TANB_INVALID_ARG, "level 0's block must be the engine block %d", e->B);
  long long off = 0;
  size_t nmax = e->B;
  lv->clear();
  for (uint32_t l = 0; l < nlevels; ++l) {
    const uint32_t N = block[l];
    if (parts[l] == 0) return efail(TANB_INVALID_ARG, "level %u has no partitions", l);
    if (l > 0) {
      if ((N & (N - 1)) || N <= block[l - 1] || N > (1u << tanb::kMaxLog2Level))
        return efail(TANB_INVALID_ARG, "level %u: block %u must be a power of two above the previous level's and "
                     "at most %u", l, N, 1u << tanb::kMaxLog2Level);
      if (off < (long long)N)
        return efail(TANB_INVALID_ARG, "level %u starts at tap %lld < its block %u (would add latency)", l, off, N);
      LevelSpec s;
      while ((1u << s.log2N) < N) ++s.log2N;
      s.K = (int)parts[l];
      s.off = off;
      s.nfl = (int)((off + N - 1) / N);
      s.Kr = s.K + s.nfl - 1;
      // Work items of a level take one bin slice per base block, so a level
      // has only ngroup of them at a time: groups of at most Q partitions,
      // and at least 8 groups when the level has 16 or more partitions, so
      // that a level with few channels still spreads over many warps.
      s.q = std::max(2, std::min(e->Q, (s.K - 2 + 7) / 8));
      s.ngroup = s.K > 2 ? (s.K - 2 + s.q - 1) / s.q : 0;
      s.R = (int)pow2_at_least((size_t)off + N + 2 * (size_t)e->B);
      lv->push_back(s);
      nmax = std::max<size_t>(nmax, N);
    } else {
      *P0 = (int)parts[0];
    }
    off += (long long)N * parts[l];
  }
  if (off < (long long)ir_length) return efail(TANB_INVALID_ARG, "levels cover %lld < %u taps", off, ir_length);
  *rin = (int)pow2_at_least(2 * nmax + e->B);
  return TANB_OK;
}

// Grows the work-item table to hold at least `need` more items (a new device
// table and pinned mirror with the old contents; the graphs, which hold the
// table's address, are rebuilt on their next use). Caller holds mu and has
// drained the audio stream.
cudaError_t grow_items(tanb_engine* e, size_t need) {
  const size_t cap = std::max(2 * e->max_items, e->max_items + need);
  EngItem* d = nullptr;
  EngItem* h = nullptr;
  cudaError_t r = cudaMalloc(&d, cap * sizeof(EngItem));
  if (r == cudaSuccess) r = cudaMallocHost(&h, cap * sizeof(EngItem));
  if (r != cudaSuccess) {
    cudaFree(d);
    cudaFreeHost(h);
    return r;
  }
  std::memcpy(h, e->h_items, e->max_items * sizeof(EngItem));
  for (size_t i = e->max_items; i < cap; ++i) h[i] = EngItem{-1, 0, 0, 0, -1, 0};
  r = cudaMemcpyAsync(d, h, cap * sizeof(EngItem), cudaMemcpyHostToDevice, e->stream);
  if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
  if (r != cudaSuccess) {
    cudaFree(d);
    cudaFreeHost(h);
    return r;
  }
  cudaFree(e->d_items);
  cudaFreeHost(e->h_items);
  e->d_items = d;
  e->h_items = h;
  e->max_items = cap;
  e->item_alloc.grow(cap);
  return cudaSuccess;
}

int32_t open_session(tanb_engine* e, uint32_t channels, uint32_t ir_length, uint32_t nlevels,
                     const uint32_t* level_block, const uint32_t* level_parts, int32_t* session,
                     uint32_t* first_slot) {
  tanb::NvtxRange range("tanb engine open session");
  if (!e || !session) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  if (channels == 0 || ir_length == 0) return efail(TANB_INVALID_ARG, "channels and IR length must be > 0");
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  Session s;
  s.C = (int)channels;
  s.L = (int)ir_length;
  if (nlevels) {
    const int32_t r = make_levels(e, ir_length, nlevels, level_block, level_parts, &s.lv, &s.P, &s.rin);
    if (r != TANB_OK) return r;
  } else {
    s.P = (int)std::max<uint32_t>(1, (ir_length + e->B - 1) / e->B);
  }
  // work items cover partitions [2, P); the head does partitions 0 and 1
  s.nitem = s.P > 2 ? (s.P - 2 + e->Q - 1) / e->Q : 0;
  s.items_per_chan = 2 * s.nitem;  // two halves of the bins per partition group
  for (const LevelSpec& l : s.lv) s.items_per_chan += l.ngroup;
  const size_t per_chan = chan_bytes(e, s.P, s.nitem, s.lv, s.rin);
  s.arena_bytes = per_chan * s.C;
  if (!e->arena_alloc.alloc(s.arena_bytes / kAlign, &s.arena_off))
    return efail(TANB_OUT_OF_MEMORY, "session of %u channels x %u taps needs %zu bytes; device budget exhausted",
                 channels, ir_length, s.arena_bytes);
  if (!e->slot_alloc.alloc(s.C, &s.slot0)) {
    e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
    return efail(TANB_OUT_OF_MEMORY, "no %u free channel slots", channels);
  }
  const size_t nit_total = (size_t)s.C * s.items_per_chan;
  if (nit_total && !e->item_alloc.alloc(nit_total, &s.item0)) {
    cudaError_t r = cudaStreamSynchronize(e->stream);
    if (r == cudaSuccess) r = grow_items(e, nit_total);
    if (r != cudaSuccess || !e->item_alloc.alloc(nit_total, &s.item0)) {
      e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
      e->slot_alloc.release(s.slot0, s.C);
      return efail(TANB_OUT_OF_MEMORY, "work-item table full");
    }
  }
  s.lv_first.assign(s.lv.size(), 0);
  for (size_t l = 0; l < s.lv.size(); ++l) {
    const int c = level_class(e, s.lv[l].log2N);
    if (!e->lvl_alloc[c].alloc(s.C, &s.lv_first[l])) {
      for (size_t m = 0; m < l; ++m) e->lvl_alloc[level_class(e, s.lv[m].log2N)].release(s.lv_first[m], s.C);
      e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
      e->slot_alloc.release(s.slot0, s.C);
      if (nit_total) e->item_alloc.release(s.item0, nit_total);
      return efail(TANB_OUT_OF_MEMORY, "level table full");
    }
  }
  // the new session's memory is cleared on the audio stream, after every
  // block already queued there (which may still read a closed session's data
  // in the same range)
  char* base = e->arena + s.arena_off * kAlign;
  ENG_CUDA(cudaMemsetAsync(base, 0, s.arena_bytes, e->stream));
  const size_t B = e->B;
  std::vector<EngNu> nus(s.lv.empty() ? 0 : s.C);
  std::vector<EngNu*> nu_dev(nus.size());
  s.zero.assign(s.C, {});
  for (int j = 0; j < s.C; ++j) {
    auto& zero = s.zero[j];
    EngChan ch{};
    ch.H = base;
    base += align_up(2 * (size_t)s.P * B * spec_bytes(e->spec));
    if (spec_scaled(e->spec)) {
      ch.scale = reinterpret_cast<float*>(base);
      base += align_up(2 * (size_t)s.P * 4);
    }
    // delay line, history and partial sums are consecutive: one flush range
    char* z0 = base;
    ch.fdl = reinterpret_cast<float2*>(base);
    base += align_up((size_t)s.P * B * fdl_bytes(e->spec));
    ch.prev = reinterpret_cast<float*>(base);
    base += align_up(B * 4);
    ch.part = reinterpret_cast<float2*>(base);
    base += align_up(4 * (size_t)s.nitem * B * 8);
    zero.push_back({z0, (size_t)(base - z0)});
    ch.P = s.P;
    ch.nitem = s.nitem;
    ch.cur = 0;
    ch.active = 0;
    ch.pending = 0;
    ch.run = 1;
    const int slot = (int)(s.slot0 + j);
    size_t it = s.item0 + (size_t)j * s.items_per_chan;
    for (int r = 0; r < s.nitem; ++r) {
      const int i0 = 2 + r * e->Q;
      for (int half = 0; half < 2; ++half)
        e->h_items[it++] = EngItem{slot, i0, std::min(s.P, i0 + e->Q), r, -1, half};
    }
    if (!s.lv.empty()) {
      EngNu& nu = nus[j];
      nu_dev[j] = reinterpret_cast<EngNu*>(base);
      ch.nu = nu_dev[j];
      base += align_up(sizeof(EngNu));
      nu.in_ring = reinterpret_cast<float*>(base);
      nu.rin = s.rin;
      nu.nlv = (int)s.lv.size();
      zero.push_back({base, (size_t)s.rin * 4});
      base += align_up((size_t)s.rin * 4);
      for (size_t l = 0; l < s.lv.size(); ++l) {
        const LevelSpec& ls = s.lv[l];
        const size_t N = (size_t)1 << ls.log2N;
        const int c = level_class(e, ls.log2N);
        const size_t rec = (size_t)c * e->max_channels + s.lv_first[l] + j;
        EngLevel lv{};
        lv.H = base;
        base += align_up(2 * (size_t)ls.K * N * spec_bytes(e->spec));
        if (spec_scaled(e->spec)) {
          lv.scale = reinterpret_cast<float*>(base);
          base += align_up(2 * (size_t)ls.K * 4);
        }
        char* z1 = base;
        lv.fdl = reinterpret_cast<float2*>(base);
        base += align_up((size_t)ls.Kr * N * fdl_bytes(e->spec));
        lv.part = reinterpret_cast<float2*>(base);
        base += align_up(2 * (size_t)ls.ngroup * N * 8);
        lv.ring = reinterpret_cast<float*>(base);
        base += align_up(2 * (size_t)ls.R * 4);
        zero.push_back({z1, (size_t)(base - z1)});
        lv.chan = slot;
        lv.log2N = ls.log2N;
        lv.K = ls.K;
        lv.Kr = ls.Kr;
        lv.ngroup = ls.ngroup;
        lv.R = ls.R;
        lv.off = ls.off;
        e->h_levels[rec] = lv;
        nu.ring[l] = lv.ring;
        nu.R[l] = ls.R;
        for (int g = 0; g < ls.ngroup; ++g) {
          const int i0 = 2 + g * ls.q;
          e->h_items[it++] = EngItem{slot, i0, std::min(ls.K, i0 + ls.q), g, (int)(c * e->max_channels +
                                     s.lv_first[l] + j), 0};
        }
      }
    }
    e->h_chans[slot] = ch;
  }
  if (base != e->arena + s.arena_off * kAlign + s.arena_bytes)
    return efail(TANB_FAIL, "session layout does not match its size (internal error)");
  // table uploads from staging (the mirrors keep changing under the audio path)
  ENG_CUDA(begin_stage(e, nus.size() * (sizeof(EngNu) + 16) + s.lv.size() * s.C * sizeof(EngLevel) + 16 * s.lv.size() +
                              s.C * sizeof(EngChan) + nit_total * sizeof(EngItem) + 64));
  for (size_t j = 0; j < nus.size(); ++j) ENG_CUDA(stage_copy(e, nu_dev[j], &nus[j], sizeof(EngNu)));
  for (size_t l = 0; l < s.lv.size(); ++l) {
    const size_t first = (size_t)level_class(e, s.lv[l].log2N) * e->max_channels + s.lv_first[l];
    ENG_CUDA(stage_copy(e, e->d_levels + first, e->h_levels + first, s.C * sizeof(EngLevel)));
  }
  ENG_CUDA(stage_copy(e, e->d_chans + s.slot0, e->h_chans + s.slot0, s.C * sizeof(EngChan)));
  ENG_CUDA(stage_copy(e, e->d_items + s.item0, e->h_items + s.item0, nit_total * sizeof(EngItem)));
  ENG_CUDA(end_stage(e));
  ENG_CUDA(cudaEventCreateWithFlags(&s.staged_ev, cudaEventDisableTiming));
  s.staged_mask.assign(s.C, 0);
  s.id = e->next_id++;
  e->sessions[s.id] = s;
  update_hwm(e);
  *session = s.id;
  if (first_slot) *first_slot = (uint32_t)s.slot0;
  return TANB_OK;
}

int32_t engine_update(tanb_engine* e, int32_t session, const float* const* ir, size_t n, bool device, uint32_t op,
                      const uint8_t* mask) {
  tanb::NvtxRange range("tanb engine IR update");
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  if (!ir) return efail(TANB_INVALID_ARG, "ppBuffer == NULL");
  std::lock_guard<std::mutex> ulock(e->upd_mu);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  // the previous upload's copies read the pinned staging rewritten below
  ENG_CUDA(cudaStreamSynchronize(e->upd_stream));
  Session s;
  std::vector<int> chans;  // session channels updated
  {
    // read the session and choose the idle IR slots under the main lock: the
    // audio path flips slots only under this lock, so the choice is consistent
    std::lock_guard<std::mutex> lock(e->mu);
    auto it = e->sessions.find(session);
    if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
    s = it->second;
    if (n > (size_t)s.L) return efail(TANB_INVALID_ARG, "IR length %zu exceeds the session's %d", n, s.L);
    for (int j = 0; j < s.C; ++j) {
      if (mask && !mask[j]) continue;
      if (!ir[j] && n) return efail(TANB_INVALID_ARG, "ppBuffer[%d] == NULL", j);
      chans.push_back(j);
    }
    if (chans.empty()) return TANB_OK;
    for (size_t q = 0; q < chans.size(); ++q) {
      const int j = chans[q];
      e->h_upd[q] = EngUpd{(int)(s.slot0 + j), 1 - e->h_chans[s.slot0 + j].active, nullptr, (int64_t)n};
    }
    it->second.staged = false;  // a newer upload supersedes one not yet committed
    // The mirror (and so the idle-slot choice) already reflects every block
    // enqueued on the audio stream; blocks still running there may read the
    // chosen slot (a crossfade from it), so the transform waits for them.
    ENG_CUDA(cudaEventRecord(e->ev_audio, e->stream));
    ENG_CUDA(cudaStreamWaitEvent(e->upd_stream, e->ev_audio, 0));
  }
  const int nch = (int)chans.size();
  if (!device && n) {
    const size_t need = n * (size_t)nch;
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
  }
  if (device) {
    // the transforms read the caller's rows in place
    for (int q = 0; q < nch; ++q) e->h_upd[q].src = ir[chans[q]];
  } else if (n) {
    // compact staging (row stride n) copied on the host pool, one transfer
    auto copy_row = [&](int q) { tanb::copy_for_device(e->h_ir + (size_t)q * n, ir[chans[q]], n * sizeof(float)); };
    if ((size_t)nch * n * sizeof(float) >= (1u << 20))
      tanb::host_parallel_for(nch, copy_row);
    else
      for (int q = 0; q < nch; ++q) copy_row(q);
    ENG_CUDA(cudaMemcpyAsync(e->d_ir, e->h_ir, (size_t)nch * n * sizeof(float), cudaMemcpyHostToDevice,
                             e->upd_stream));
    for (int q = 0; q < nch; ++q) e->h_upd[q].src = e->d_ir + (size_t)q * n;
  }
  ENG_CUDA(cudaMemcpyAsync(e->d_upd, e->h_upd, nch * sizeof(EngUpd), cudaMemcpyHostToDevice, e->upd_stream));
  ENG_CUDA(tanb::eng_launch_ir(e->log2B, e->spec, e->d_chans, e->d_upd, nch, s.P, e->d_tw, e->upd_stream));
  // the levels of a non-uniform session, one transform launch per level
  for (size_t l = 0; l < s.lv.size(); ++l) {
    const int c = level_class(e, s.lv[l].log2N);
    EngLvlUpd* hl = e->h_lupd + l * e->max_channels;
    for (int q = 0; q < nch; ++q)
      hl[q] = EngLvlUpd{(int)(s.lv_first[l] + chans[q]), e->h_upd[q].slot, e->h_upd[q].src, (int64_t)n};
    EngLvlUpd* dl = e->d_lupd + l * e->max_channels;
    ENG_CUDA(cudaMemcpyAsync(dl, hl, nch * sizeof(EngLvlUpd), cudaMemcpyHostToDevice, e->upd_stream));
    ENG_CUDA(tanb::eng_launch_level_ir(s.lv[l].log2N, e->spec, e->d_levels + (size_t)c * e->max_channels, dl, nch,
                                       s.lv[l].K, e->d_tw_lv[c], e->upd_stream));
  }
  ENG_CUDA(cudaEventRecord(s.staged_ev, e->upd_stream));
  // BLOCK_UNTIL_READY: the new IR is ready for the next block when this returns
  if (op & TANB_OPERATION_FLAG_BLOCK_UNTIL_READY) ENG_CUDA(cudaEventSynchronize(s.staged_ev));
  {
    std::lock_guard<std::mutex> lock(e->mu);
    auto it = e->sessions.find(session);
    if (it != e->sessions.end()) {
      it->second.staged = true;
      std::fill(it->second.staged_mask.begin(), it->second.staged_mask.end(), 0);
      for (int j : chans) it->second.staged_mask[j] = 1;
    }
    e->n_ir += 1;
  }
  return TANB_OK;
}

// One block: commit staged updates, then the block (a graph for the host
// buffers, direct launches for other rows). Caller holds mu.
int32_t run_block(tanb_engine* e, const tanb::EngRows* rows) {
  Clock::time_point t0 = Clock::now();
  ENG_CUDA(commit_updates(e));
  e->bt_commit = us_since(t0);
  const unsigned due = due_mask(e, e->k_host);
  if (!rows) {
    cudaGraphExec_t ge = nullptr;
    e->bt_build = 0;
    ENG_CUDA(ensure_graph(e, due, &ge));
    t0 = Clock::now();
    ENG_CUDA(cudaGraphLaunch(ge, e->stream));
    e->bt_launch = us_since(t0);
  } else {
    if (e->profiling) ENG_CUDA(cudaEventRecord(e->pa, e->stream));
    ENG_CUDA(enqueue_block(e, *rows, due));
    if (e->profiling) {
      ENG_CUDA(cudaEventRecord(e->pb, e->stream));
      ENG_CUDA(cudaEventSynchronize(e->pb));
      float a = 0;
      cudaEventElapsedTime(&a, e->pa, e->pb);
      e->ms_block += a;
      e->n_timed += 1;
    }
  }
  e->n_block += 1;
  advance_mirror(e);
  return TANB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Internal interface for the drop-in object's non-uniform methods
// (tanb_engine_host.h).
namespace tanb {

int32_t engine_update_channels(tanb_engine* e, int32_t session, const float* const* ir, size_t n, bool device,
                               uint32_t op, const uint8_t* mask) {
  return engine_update(e, session, ir, n, device, op, mask);
}

int32_t engine_flush_channel(tanb_engine* e, int32_t session, int channel) {
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->sessions.find(session);
  if (it == e->sessions.end() || channel < 0 || channel >= it->second.C)
    return efail(TANB_INVALID_ARG, "no channel %d in session %d", channel, session);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  for (const auto& z : it->second.zero[channel]) ENG_CUDA(cudaMemsetAsync(z.first, 0, z.second, e->stream));
  return TANB_OK;
}

size_t engine_nu_session_bytes(int block, int spectrum, int channels, uint32_t ir_length, uint32_t nlevels,
                               const uint32_t* level_block, const uint32_t* level_parts) {
  uint64_t bytes = 0;
  if (tanb_engine_session_bytes((uint32_t)block, (uint32_t)spectrum, 0, (uint32_t)channels, ir_length, nlevels,
                                level_block, level_parts, &bytes) != TANB_OK)
    return 0;
  return (size_t)bytes;
}

int32_t engine_process_rows(tanb_engine* e, const EngRows& rows) {
  std::lock_guard<std::mutex> lock(e->mu);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  if (e->sessions.empty()) return efail(TANB_WRONG_STATE, "no open sessions");
  return run_block(e, &rows);
}

}  // namespace tanb

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
  // work items: 64 per channel slot to start with; the table grows when a
  // session needs more (non-uniform levels take one item per bin slice)
  e->max_items = (size_t)max_channels * 64;
  e->nclass = tanb::kMaxLog2Level - e->log2B;
  cudaError_t r = cudaSetDevice(ctx->device);
  if (r == cudaSuccess) r = tanb::eng_prepare();
  // the audio streams at the device's highest priority, IR uploads at its
  // lowest: when both have CTAs waiting for an SM, the block's go first
  int prio_low = 0, prio_high = 0;
  if (r == cudaSuccess) r = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (r == cudaSuccess) r = cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, prio_high);
  // the level heads of each size class on a stream of their own, so that the
  // classes due at one block run side by side
  e->lstreams.assign(e->nclass, nullptr);
  e->ev_joins.assign(e->nclass, nullptr);
  for (int c = 0; c < e->nclass && r == cudaSuccess; ++c) {
    r = cudaStreamCreateWithPriority(&e->lstreams[c], cudaStreamNonBlocking, prio_high);
    if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_joins[c], cudaEventDisableTiming);
  }
  if (r == cudaSuccess) r = cudaStreamCreateWithPriority(&e->upd_stream, cudaStreamNonBlocking, prio_low);
  const size_t io = e->max_channels * e->B;
  const size_t nlev = (size_t)e->nclass * e->max_channels;
  if (r == cudaSuccess) r = cudaMalloc(&e->arena, std::max<size_t>(budget_bytes, kAlign));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_chans, e->max_channels * sizeof(EngChan));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_items, e->max_items * sizeof(EngItem));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_levels, std::max<size_t>(1, nlev) * sizeof(EngLevel));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_block, 2 * sizeof(long long));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_upd, e->max_channels * sizeof(EngUpd));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_lupd, tanb::kMaxLevels * e->max_channels * sizeof(EngLvlUpd));
  if (r == cudaSuccess) r = cudaMalloc(&e->d_tw, 2 * e->B * sizeof(float2));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_chans, e->max_channels * sizeof(EngChan));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_items, e->max_items * sizeof(EngItem));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_levels, std::max<size_t>(1, nlev) * sizeof(EngLevel));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_in, io * sizeof(float));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_out, io * sizeof(float));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_upd, e->max_channels * sizeof(EngUpd));
  if (r == cudaSuccess) r = cudaMallocHost(&e->h_lupd, tanb::kMaxLevels * e->max_channels * sizeof(EngLvlUpd));
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_audio, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_stage, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_upd_done, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreate(&e->pa);
  if (r == cudaSuccess) r = cudaEventCreate(&e->pb);
  e->d_tw_lv.assign(e->nclass, nullptr);
  for (int c = 0; c < e->nclass && r == cudaSuccess; ++c)
    r = cudaMalloc(&e->d_tw_lv[c], (size_t)(4 << (e->log2B + c)) * sizeof(float2));  // 2N entries
  if (r != cudaSuccess) {
    free_engine(e);
    delete e;
    cudaGetLastError();
    return efail(r == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, "engine setup: %s",
                 cudaGetErrorString(r));
  }
  std::memset(e->h_chans, 0, e->max_channels * sizeof(EngChan));
  for (size_t i = 0; i < e->max_items; ++i) e->h_items[i] = EngItem{-1, 0, 0, 0, -1, 0};
  for (size_t i = 0; i < nlev; ++i) {
    e->h_levels[i] = EngLevel{};
    e->h_levels[i].chan = -1;
  }
  std::memset(e->h_in, 0, io * sizeof(float));
  std::memset(e->h_out, 0, io * sizeof(float));
  e->arena_alloc.reset(budget_bytes / kAlign);
  e->slot_alloc.reset(e->max_channels);
  e->item_alloc.reset(e->max_items);
  e->lvl_alloc.assign(e->nclass, RangeAlloc());
  for (auto& a : e->lvl_alloc) a.reset(e->max_channels);
  e->lvl_hwm.assign(e->nclass, 0);
  std::vector<float2> tw(2 * e->B);
  tanb::make_twiddles(2 * e->B, tw.data());
  r = cudaMemcpy(e->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
  for (int c = 0; c < e->nclass && r == cudaSuccess; ++c) {
    std::vector<float2> twl((size_t)4 << (e->log2B + c));
    tanb::make_twiddles((int)twl.size(), twl.data());
    r = cudaMemcpy(e->d_tw_lv[c], twl.data(), twl.size() * sizeof(float2), cudaMemcpyHostToDevice);
  }
  if (r == cudaSuccess) r = cudaMemsetAsync(e->d_chans, 0, e->max_channels * sizeof(EngChan), e->stream);
  if (r == cudaSuccess) r = upload_items(e, 0, e->max_items);
  if (r == cudaSuccess) r = upload_levels(e, 0, nlev);
  if (e->d_block) e->d_done = reinterpret_cast<unsigned int*>(e->d_block + 1);
  if (r == cudaSuccess) r = cudaMemsetAsync(e->d_block, 0, 2 * sizeof(long long), e->stream);
  if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
  // tail CTAs of the block launch: as many as fit on the GPU at once (B / 4
  // threads each at up to 64 registers: 1024 threads per SM)
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int per_sm = std::max(1, std::min(32, 1024 / (e->B / 4)));
  e->tail_grid = e->sms * per_sm;
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

int32_t tanb_engine_session_bytes(uint32_t block, uint32_t spectrum, uint32_t partitions_per_item, uint32_t channels,
                                  uint32_t ir_length, uint32_t nlevels, const uint32_t* level_block,
                                  const uint32_t* level_parts, uint64_t* bytes) {
  if (!bytes) return efail(TANB_INVALID_POINTER, "null argument");
  *bytes = 0;
  if (block < 128 || block > 2048 || (block & (block - 1)) || spectrum > tanb::kSpecFP24 || channels == 0 ||
      ir_length == 0)
    return efail(TANB_INVALID_ARG, "invalid engine block, spectrum, channels or IR length");
  if (nlevels && (!level_block || !level_parts)) return efail(TANB_INVALID_POINTER, "null level schedule");
  tanb_engine probe;  // shape only: no device state
  probe.B = (int)block;
  while ((1 << probe.log2B) < probe.B) ++probe.log2B;
  probe.spec = (int)spectrum;
  probe.Q = partitions_per_item ? (int)partitions_per_item : 32;
  std::vector<LevelSpec> lv;
  int P = 0, rin = 0;
  if (nlevels) {
    const int32_t r = make_levels(&probe, ir_length, nlevels, level_block, level_parts, &lv, &P, &rin);
    if (r != TANB_OK) return r;
  } else {
    P = (int)std::max<uint32_t>(1, (ir_length + block - 1) / block);
  }
  const int nitem = P > 2 ? (P - 2 + probe.Q - 1) / probe.Q : 0;
  *bytes = (uint64_t)chan_bytes(&probe, P, nitem, lv, rin) * channels;
  return TANB_OK;
}

int32_t tanb_engine_open_session(tanb_engine* e, uint32_t channels, uint32_t ir_length, int32_t* session,
                                 uint32_t* first_slot) {
  return open_session(e, channels, ir_length, 0, nullptr, nullptr, session, first_slot);
}

int32_t tanb_engine_open_session_nu(tanb_engine* e, uint32_t channels, uint32_t ir_length, uint32_t nlevels,
                                    const uint32_t* level_block, const uint32_t* level_parts, int32_t* session,
                                    uint32_t* first_slot) {
  if (!level_block || !level_parts || nlevels == 0) return efail(TANB_INVALID_POINTER, "null level schedule");
  return open_session(e, channels, ir_length, nlevels, level_block, level_parts, session, first_slot);
}

int32_t tanb_engine_close_session(tanb_engine* e, int32_t session) {
  tanb::NvtxRange range("tanb engine close session");
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> ulock(e->upd_mu);  // no IR upload may still write this session's memory
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->sessions.find(session);
  if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  // No host wait: the audio stream waits for the update stream's work queued
  // so far (an IR transform may still write this session's memory), and every
  // later use of the freed memory, slots and table rows (a new session's
  // clear and uploads) is queued on the audio stream after the blocks that
  // still read them.
  ENG_CUDA(cudaEventRecord(e->ev_upd_done, e->upd_stream));
  ENG_CUDA(cudaStreamWaitEvent(e->stream, e->ev_upd_done, 0));
  const Session s = it->second;
  if (s.staged_ev) cudaEventDestroy(s.staged_ev);
  for (int j = 0; j < s.C; ++j) e->h_chans[s.slot0 + j] = EngChan{};
  const size_t nit_total = (size_t)s.C * s.items_per_chan;
  for (size_t i = 0; i < nit_total; ++i) e->h_items[s.item0 + i] = EngItem{-1, 0, 0, 0, -1, 0};
  ENG_CUDA(begin_stage(e, s.lv.size() * (s.C * sizeof(EngLevel) + 16) + s.C * sizeof(EngChan) +
                              nit_total * sizeof(EngItem) + 64));
  for (size_t l = 0; l < s.lv.size(); ++l) {
    const size_t first = (size_t)level_class(e, s.lv[l].log2N) * e->max_channels + s.lv_first[l];
    for (int j = 0; j < s.C; ++j) {
      e->h_levels[first + j] = EngLevel{};
      e->h_levels[first + j].chan = -1;
    }
    ENG_CUDA(stage_copy(e, e->d_levels + first, e->h_levels + first, s.C * sizeof(EngLevel)));
  }
  ENG_CUDA(stage_copy(e, e->d_chans + s.slot0, e->h_chans + s.slot0, s.C * sizeof(EngChan)));
  ENG_CUDA(stage_copy(e, e->d_items + s.item0, e->h_items + s.item0, nit_total * sizeof(EngItem)));
  ENG_CUDA(end_stage(e));
  e->arena_alloc.release(s.arena_off, s.arena_bytes / kAlign);
  e->slot_alloc.release(s.slot0, s.C);
  if (nit_total) e->item_alloc.release(s.item0, nit_total);
  for (size_t l = 0; l < s.lv.size(); ++l) e->lvl_alloc[level_class(e, s.lv[l].log2N)].release(s.lv_first[l], s.C);
  e->sessions.erase(it);
  update_hwm(e);
  return TANB_OK;
}

// ---------------------------------------------------------------------------
// Session snapshot and restore (uniformly partitioned sessions): the session's
// arena range (both IR slots' spectra with their scales, delay lines, input
// history, partial-sum rows), each channel's delay-line position and IR slot,
// the session's block count and a staged IR update not yet in effect. Another
// engine with the same block, spectrum and work-item size (on this GPU or
// another) opens a session from it whose output continues bit for bit. The
// partial-sum rows are indexed by the parity of the engine's block counter;
// when the two engines' parities differ the restore swaps the halves.
// ---------------------------------------------------------------------------
namespace {

struct SessSnapHeader {
  char magic[8];
  uint32_t B, spec, Q, C, L, P, nitem, next_parity;
  uint32_t staged, pad;
  uint64_t arena_bytes;
  int64_t blocks, last_swap_block;
};
constexpr char kSessSnapMagic[8] = {'T', 'A', 'N', 'B', 'E', 'S', 'N', '1'};

size_t sess_snap_bytes(const Session& s) {
  return sizeof(SessSnapHeader) + (size_t)s.C * (3 * sizeof(int32_t) + 1) + s.arena_bytes;
}

// Offset of a channel's partial-sum rows within its arena bytes (the layout
// open_session lays down).
size_t part_offset(const tanb_engine* e, int P) {
  const size_t B = e->B;
  size_t off = align_up(2 * (size_t)P * B * spec_bytes(e->spec));
  if (spec_scaled(e->spec)) off += align_up(2 * (size_t)P * 4);
  off += align_up((size_t)P * B * fdl_bytes(e->spec));
  off += align_up(B * 4);
  return off;
}

}  // namespace

int32_t tanb_engine_session_snapshot_bytes(tanb_engine* e, int32_t session, uint64_t* bytes) {
  if (bytes) *bytes = 0;
  if (!e || !bytes) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->sessions.find(session);
  if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
  if (!it->second.lv.empty()) return efail(TANB_NOT_SUPPORTED, "snapshots cover uniformly partitioned sessions");
  *bytes = sess_snap_bytes(it->second);
  return TANB_OK;
}

int32_t tanb_engine_session_snapshot(tanb_engine* e, int32_t session, void* buffer, uint64_t bytes) {
  if (!e || !buffer) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> ulock(e->upd_mu);  // no IR upload may still write the session's memory
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->sessions.find(session);
  if (it == e->sessions.end()) return efail(TANB_INVALID_ARG, "no session %d", session);
  const Session& s = it->second;
  if (!s.lv.empty()) return efail(TANB_NOT_SUPPORTED, "snapshots cover uniformly partitioned sessions");
  if (bytes < sess_snap_bytes(s))
    return efail(TANB_INVALID_ARG, "snapshot buffer of %llu bytes, %zu needed", (unsigned long long)bytes,
                 sess_snap_bytes(s));
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  ENG_CUDA(cudaStreamSynchronize(e->upd_stream));
  ENG_CUDA(cudaStreamSynchronize(e->stream));
  for (cudaStream_t ls : e->lstreams) ENG_CUDA(cudaStreamSynchronize(ls));
  char* p = static_cast<char*>(buffer);
  SessSnapHeader h{};
  std::memcpy(h.magic, kSessSnapMagic, sizeof(h.magic));
  h.B = (uint32_t)e->B;
  h.spec = (uint32_t)e->spec;
  h.Q = (uint32_t)e->Q;
  h.C = (uint32_t)s.C;
  h.L = (uint32_t)s.L;
  h.P = (uint32_t)s.P;
  h.nitem = (uint32_t)s.nitem;
  // the next block's heads read the partial rows of this parity
  h.next_parity = (uint32_t)(e->k_host & 1);
  h.staged = s.staged ? 1u : 0u;
  h.arena_bytes = s.arena_bytes;
  h.blocks = s.blocks;
  h.last_swap_block = s.last_swap_block;
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  for (int j = 0; j < s.C; ++j) {
    const EngChan& ch = e->h_chans[s.slot0 + j];
    const int32_t v[3] = {ch.cur, ch.active, ch.pending};
    std::memcpy(p, v, sizeof(v));
    p += sizeof(v);
  }
  for (int j = 0; j < s.C; ++j) *p++ = (char)(s.staged && s.staged_mask[j] ? 1 : 0);
  ENG_CUDA(cudaMemcpy(p, e->arena + s.arena_off * kAlign, s.arena_bytes, cudaMemcpyDeviceToHost));
  return TANB_OK;
}

int32_t tanb_engine_open_session_restore(tanb_engine* e, const void* buffer, uint64_t bytes, int32_t* session,
                                         uint32_t* first_slot) {
  if (!e || !buffer || !session) return efail(TANB_INVALID_POINTER, "null argument");
  *session = -1;
  if (bytes < sizeof(SessSnapHeader)) return efail(TANB_INVALID_ARG, "not a session snapshot");
  const char* p = static_cast<const char*>(buffer);
  SessSnapHeader h;
  std::memcpy(&h, p, sizeof(h));
  p += sizeof(h);
  if (std::memcmp(h.magic, kSessSnapMagic, sizeof(h.magic)) != 0) return efail(TANB_INVALID_ARG, "not a session snapshot");
  if (h.B != (uint32_t)e->B || h.spec != (uint32_t)e->spec || h.Q != (uint32_t)e->Q)
    return efail(TANB_INVALID_ARG, "snapshot of an engine with block %u, spectrum %u, %u partitions per item", h.B,
                 h.spec, h.Q);
  if (h.C == 0 || h.L == 0 || bytes < sizeof(SessSnapHeader) + (size_t)h.C * 13 + h.arena_bytes)
    return efail(TANB_INVALID_ARG, "short or corrupt session snapshot");
  int32_t sid = -1;
  uint32_t slot0 = 0;
  int32_t r = open_session(e, h.C, h.L, 0, nullptr, nullptr, &sid, &slot0);
  if (r != TANB_OK) return r;
  bool match;
  {
    std::lock_guard<std::mutex> lock(e->mu);
    const Session& s = e->sessions[sid];
    match = (uint32_t)s.P == h.P && (uint32_t)s.nitem == h.nitem && s.arena_bytes == h.arena_bytes;
  }
  if (!match) {
    tanb_engine_close_session(e, sid);
    return efail(TANB_INVALID_ARG, "snapshot layout does not match this engine's");
  }
  std::lock_guard<std::mutex> lock(e->mu);
  Session& s = e->sessions[sid];
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  const char* chan_state = p;
  p += (size_t)h.C * 3 * sizeof(int32_t);
  const char* staged_mask = p;
  p += h.C;
  // the arena bytes, with the partial-sum halves exchanged when this engine's
  // next block has the other parity
  std::vector<char> arena(p, p + h.arena_bytes);
  if (h.next_parity != (uint32_t)(e->k_host & 1) && s.nitem > 0) {
    const size_t per = s.arena_bytes / s.C, half = 2 * (size_t)s.nitem * e->B * sizeof(float2);
    const size_t off = part_offset(e, s.P);
    for (int j = 0; j < s.C; ++j) {
      char* a = arena.data() + j * per + off;
      std::swap_ranges(a, a + half, a + half);
    }
  }
  // the session's clear and table uploads are queued on the audio stream: the
  // copy goes after them
  ENG_CUDA(cudaStreamSynchronize(e->stream));
  ENG_CUDA(cudaMemcpy(e->arena + s.arena_off * kAlign, arena.data(), s.arena_bytes, cudaMemcpyHostToDevice));
  for (uint32_t j = 0; j < h.C; ++j) {
    int32_t v[3];
    std::memcpy(v, chan_state + j * sizeof(v), sizeof(v));
    EngChan& ch = e->h_chans[s.slot0 + j];
    ch.cur = ((v[0] % s.P) + s.P) % s.P;
    ch.active = v[1] & 1;
    ch.pending = v[2] & 1;
  }
  ENG_CUDA(begin_stage(e, h.C * sizeof(EngChan) + 64));
  ENG_CUDA(stage_copy(e, e->d_chans + s.slot0, e->h_chans + s.slot0, h.C * sizeof(EngChan)));
  ENG_CUDA(end_stage(e));
  s.blocks = h.blocks;
  s.last_swap_block = h.last_swap_block;
  if (h.staged) {
    // an IR already transformed into the idle slot: it takes effect on the
    // next block, as it would have on the source engine
    s.staged = true;
    for (uint32_t j = 0; j < h.C; ++j) s.staged_mask[j] = staged_mask[j] ? 1 : 0;
    ENG_CUDA(cudaEventRecord(s.staged_ev, e->stream));
  }
  *session = sid;
  if (first_slot) *first_slot = slot0;
  return TANB_OK;
}

int32_t tanb_engine_update_response_td(tanb_engine* e, int32_t session, const float* const* ir, size_t n,
                                       uint32_t operationFlags) {
  return engine_update(e, session, ir, n, false, operationFlags, nullptr);
}

int32_t tanb_engine_update_response_td_device(tanb_engine* e, int32_t session, const float* const* ir,
                                              size_t n, uint32_t operationFlags) {
  return engine_update(e, session, ir, n, true, operationFlags, nullptr);
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
  tanb::NvtxRange range("tanb engine block");
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  const Clock::time_point t_call = Clock::now();
  std::lock_guard<std::mutex> lock(e->mu);
  const Clock::time_point t_locked = Clock::now();
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  if (e->sessions.empty()) return efail(TANB_WRONG_STATE, "no open sessions");
  const int32_t r = run_block(e, nullptr);
  if (r != TANB_OK) return r;
  const Clock::time_point tw = Clock::now();
  ENG_CUDA(cudaEventSynchronize(e->ev_out));
  e->bt_wait = us_since(tw);
  e->bt_lock = std::chrono::duration<double, std::micro>(t_locked - t_call).count();
  e->bt_total = us_since(t_call);
  e->bt_max = std::max(e->bt_max, e->bt_total);
  return TANB_OK;
}

int32_t tanb_engine_process_device(tanb_engine* e, const float* in, float* out, uint32_t ld) {
  tanb::NvtxRange range("tanb engine block (device rows)");
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> lock(e->mu);
  if (!out) return efail(TANB_INVALID_ARG, "null output");
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  if (e->sessions.empty()) return efail(TANB_WRONG_STATE, "no open sessions");
  tanb::EngRows rows;
  rows.in_base = in;
  rows.out_base = out;
  rows.ld = ld ? (int)ld : e->B;
  return run_block(e, &rows);
}

int32_t tanb_engine_synchronize(tanb_engine* e) {
  if (!e) return efail(TANB_INVALID_POINTER, "null engine");
  std::lock_guard<std::mutex> lock(e->mu);
  ENG_CUDA(cudaSetDevice(e->ctx->device));
  ENG_CUDA(cudaStreamSynchronize(e->upd_stream));
  ENG_CUDA(cudaStreamSynchronize(e->stream));
  destroy_retired(e);
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
    int64_t head = 4 * B * 4 + (int64_t)s.nitem * B * 8 + (s.P > 1 ? 2 * B * sb + B * xb : B * sb) + B * xb;
    // non-uniform levels, per base block on average over their periods: the
    // level items stream partitions [2, K) and write the partial rows; the
    // level head reads its frame, the partial rows, partitions 0 and 1 and
    // X_{j-1}, writes X_j and its N outputs; the base head writes the input
    // history and reads one block of every level's ring
    int64_t levels = 0;
    if (!s.lv.empty()) head += B * 4 + (int64_t)s.lv.size() * B * 4;
    for (const LevelSpec& l : s.lv) {
      const int64_t N = 1LL << l.log2N, p = N / B;
      const int64_t items = (l.K > 2 ? (int64_t)(l.K - 2) * N * (sb + xb) : 0) + (int64_t)l.ngroup * N * 8;
      const int64_t lhead = 2 * N * 4 + (int64_t)l.ngroup * N * 8 + (l.K > 1 ? 2 * N * sb + N * xb : N * sb) +
                            N * xb + N * 4;
      levels += (items + lhead) / p;
    }
    block_bytes += (int64_t)s.C * (tail + head + levels);
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

int32_t tanb_engine_block_times(tanb_engine* e, double us[8]) {
  if (!e || !us) return efail(TANB_INVALID_POINTER, "null argument");
  std::lock_guard<std::mutex> lock(e->mu);
  us[0] = e->bt_lock;
  us[1] = e->bt_commit;
  us[2] = e->bt_build;
  us[3] = e->bt_launch;
  us[4] = e->bt_wait;
  us[5] = e->bt_total;
  us[6] = e->bt_max;
  us[7] = (double)e->n_graph_builds;
  e->bt_max = 0;
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
