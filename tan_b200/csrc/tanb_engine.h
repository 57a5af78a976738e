// Internal interface of the batched engine (tanb_engine.cpp <-> tanb_engine_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tanb {

enum { kSpecFP32 = 0, kSpecFP16 = 1, kSpecBF16 = 2 };

// One channel slot of the engine's device channel table. Pointers and sizes
// are written by the host when a session opens; cur / active / pending are
// advanced by the kernels (the host keeps an exact mirror).
struct EngChan {
  void* H;        // IR spectra [2 slots][P][B], element type by spectrum kind
  float* scale;   // per-partition scales [2 slots][P] (FP16 / BF16 only)
  float2* fdl;    // delay line [P][B]; slot (cur + i) mod P holds X_{k-i}
  float* prev;    // previous input block [B] (overlap-save history)
  float2* part;   // tail partial sums [2: active IR, pending IR][nitem][B]
  int32_t P;      // partitions
  int32_t nitem;  // tail work items of this channel
  int32_t cur;    // delay-line slot of the newest spectrum
  int32_t active; // IR slot in use
  int32_t pending;  // new IR waiting in slot 1 - active (crossfade next block)
  int32_t run;    // slot belongs to an open session
  int32_t session;
  int32_t pad;
};

// A tail work item: partitions [i0, i1) of channel `chan`, partial sum row `row`.
struct EngItem {
  int32_t chan;  // -1: free
  int32_t i0, i1;
  int32_t row;
};

// One channel of an IR update: staging row j is channel `chan`'s IR, written
// into IR slot `slot`.
struct EngUpd {
  int32_t chan;
  int32_t slot;
  int64_t stride;  // floats between staging rows (P * B)
};

cudaError_t eng_prepare();
cudaError_t eng_launch_ir(int log2B, int spec, EngChan* chans, const float* ir, const EngUpd* upd, int nupd,
                          int maxP, const float2* tw, cudaStream_t st);
cudaError_t eng_launch_head(int log2B, int spec, EngChan* chans, int nslots, const float* in, float* out, int ld,
                            const float2* tw, cudaStream_t st);
cudaError_t eng_launch_tail(int log2B, int spec, const EngChan* chans, const EngItem* items, int item0,
                            int nitems, int mode, int grid, cudaStream_t st);

}  // namespace tanb
