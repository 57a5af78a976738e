// Internal interface of the batched engine (tanb_engine.cpp <-> tanb_engine_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tanb {

enum { kSpecFP32 = 0, kSpecFP16 = 1, kSpecBF16 = 2, kSpecFP24 = 3 };

// One channel slot of the engine's device channel table. Pointers and sizes
// are written by the host when a session opens; cur / active / pending are
// advanced by the kernels (the host keeps an exact mirror).
struct EngChan {
  void* H;        // IR spectra [2 slots][P][B], element type by spectrum kind
  float* scale;   // per-partition scales [2 slots][P] (FP16 / BF16 only)
  float2* fdl;    // delay line [P][B]; slot (cur + i) mod P holds X_{k-i}
  float* prev;    // previous input block [B] (overlap-save history)
  float2* part;   // tail partial sums [2: block parity][2: IR in use, new IR][nitem][B]
  int32_t P;      // partitions
  int32_t nitem;  // tail work items of this channel
  int32_t cur;    // delay-line slot of the newest spectrum
  int32_t active; // IR slot in use
  int32_t pending;  // new IR waiting in slot 1 - active (crossfade next block)
  int32_t run;    // slot belongs to an open session
  int32_t session;
  int32_t pad;
};

// A tail work item: partitions [i0, i1) (i0 >= 2; partitions 0 and 1 belong to
// the head) of channel `chan`, partial sum row `row`.
struct EngItem {
  int32_t chan;  // -1: free
  int32_t i0, i1;
  int32_t row;
};

// One channel of an IR update: channel `chan`'s new IR, read from `src`
// (samples at and after n read as zero), written into IR slot `slot`.
struct EngUpd {
  int32_t chan;
  int32_t slot;
  const float* src;
  int64_t n;
};

// Block-level counters in device memory: blocks processed (its parity selects
// the partial-sum rows) and CTAs finished in the running launch.
struct EngSync {
  long long* block;
  unsigned int* done;
};

cudaError_t eng_prepare();
cudaError_t eng_launch_ir(int log2B, int spec, EngChan* chans, const EngUpd* upd, int nupd, int maxP,
                          const float2* tw, cudaStream_t st);
// One audio block for every channel slot: nslots head CTAs plus tail_ctas
// persistent CTAs over the work items [0, nitems). in / out: slot s at s * ld
// (device or pinned host memory; in may be null).
cudaError_t eng_launch_block(int log2B, int spec, EngChan* chans, int nslots, const EngItem* items, int nitems,
                             int tail_ctas, const float* in, float* out, int ld, const float2* tw, EngSync sync,
                             cudaStream_t st);
// Sets `pending` on channel slots [first, first + n) (the values travel as
// kernel parameters, so the host mirror may change as soon as this returns).
cudaError_t eng_launch_mark_pending(EngChan* chans, int first, int n, cudaStream_t st);
// Partial sums of newly committed IRs (channels with pending set) for the
// coming block, over work items [item0, item0 + nitems).
cudaError_t eng_launch_commit(int log2B, int spec, const EngChan* chans, const EngItem* items, int item0,
                              int nitems, int grid, const long long* block, cudaStream_t st);

}  // namespace tanb
