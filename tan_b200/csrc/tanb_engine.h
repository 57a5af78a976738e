// Internal interface of the batched engine (tanb_engine.cpp <-> tanb_engine_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tanb {

enum { kSpecFP32 = 0, kSpecFP16 = 1, kSpecBF16 = 2, kSpecFP24 = 3 };

// Largest level block of a non-uniformly partitioned session (2^kMaxLog2Level
// samples: a 2N = 32768-point transform, one CTA of 1024 threads holding
// 16 complex values each, 128 KB of shared memory) and the number of levels
// above the base level a channel may have.
constexpr int kMaxLog2Level = 14;
constexpr int kMaxLevels = 8;

// A level of a non-uniformly partitioned channel above its base level: block
// N = 2^log2N (a multiple of the engine block B, larger than B), K partitions
// covering IR taps [off, off + K N), run once every p = N / B base blocks.
// Level block j (input samples [jN, (j+1)N)) completes with base block
// k = (j+1) p - 1; its head then computes the level's output for samples
// [off + jN, off + (j+1)N), which off >= N places after that base block.
struct EngLevel {
  void* H;         // IR spectra [2 slots][K][N], element type by spectrum kind
  float* scale;    // per-partition scales [2 slots][K] (FP16 / BF16 only)
  float2* fdl;     // delay line [Kr][N]: level block j's spectrum in slot Kr-1 - (j mod Kr)
  float2* part;    // partial sums [2: parity of the level block][ngroup][N]
  float* ring;     // output rings [2: IR slot][R]; sample t at t mod R
  int32_t chan;    // channel slot (-1: free record)
  int32_t log2N;
  int32_t K;       // partitions
  int32_t Kr;      // delay-line slots: K plus the blocks an IR swap recomputes
  int32_t ngroup;  // partial-sum rows (work-item groups over partitions [2, K))
  int32_t R;       // ring length, a power of two
  long long off;   // first tap of the level
};

// Per-channel extras of a non-uniformly partitioned channel: its input
// history (read by the level heads) and the output rings of its levels, summed
// in level order by the base head.
struct EngNu {
  float* in_ring;  // input samples; sample t at t mod rin
  int32_t rin;     // a power of two
  int32_t nlv;     // levels above the base level
  float* ring[kMaxLevels];
  int32_t R[kMaxLevels];
};

// One channel slot of the engine's device channel table. Pointers and sizes
// are written by the host when a session opens; cur / active / pending are
// advanced by the kernels (the host keeps an exact mirror). For a
// non-uniformly partitioned channel this is its base level (block B, P
// partitions covering taps [0, P B)) and `nu` points to its extras.
struct EngChan {
  void* H;        // IR spectra [2 slots][P][B], element type by spectrum kind
  float* scale;   // per-partition scales [2 slots][P] (FP16 / BF16 only)
  float2* fdl;    // delay line [P][B]; slot (cur + i) mod P holds X_{k-i}
  float* prev;    // previous input block [B] (overlap-save history)
  float2* part;   // tail partial sums [2: block parity][2: IR in use, new IR][nitem][B]
  const EngNu* nu;  // non-uniform extras, null for a uniformly partitioned channel
  int32_t P;      // partitions
  int32_t nitem;  // tail work items of this channel's base level
  int32_t cur;    // delay-line slot of the newest spectrum
  int32_t active; // IR slot in use
  int32_t pending;  // new IR waiting in slot 1 - active (crossfade next block)
  int32_t run;    // slot belongs to an open session
  int32_t session;
  int32_t pad;
};

// A tail work item. Base level (lvl < 0): partitions [i0, i1) (i0 >= 2;
// partitions 0 and 1 belong to the head) of channel `chan`, bins of half
// `slice` (0: [0, B/2), 1: [B/2, B)) of partial sum row `row`, every block.
// Level item (lvl >= 0, index into the level table):
// partitions [i0, i1) of that level, partial row `row`; at base block k it
// takes bin slice k mod p ([s B, (s + 1) B) of the level's N-bin rows) of
// the level block after the one completing in this period, so a level's tail
// is spread evenly over its p base blocks and every item works every block.
struct EngItem {
  int32_t chan;  // -1: free
  int32_t i0, i1;
  int32_t row;
  int32_t lvl;
  int32_t slice;  // base items: the half of the row's bins
};

// One channel of an IR update: channel `chan`'s new IR, read from `src`
// (samples at and after n read as zero), written into IR slot `slot`.
struct EngUpd {
  int32_t chan;
  int32_t slot;
  const float* src;
  int64_t n;
};

// One level of an IR update: level record `lvl` (of one size class), taps
// [off, off + K N) of `src` (zero at and after n) into IR slot `slot`.
struct EngLvlUpd {
  int32_t lvl;
  int32_t slot;
  const float* src;
  int64_t n;
};

// Block-level counters in device memory: blocks processed (its parity selects
// the partial-sum rows) and CTAs finished in the running block (over every
// kernel of the block).
struct EngSync {
  long long* block;
  unsigned int* done;
};

// Per-channel input / output rows of a block launch: slot s reads
// in_tab[s] (or in_base + s * ld) and writes out_tab[s] (or out_base + s * ld).
// A null row reads as silence / discards the output.
struct EngRows {
  const float* in_base = nullptr;
  float* out_base = nullptr;
  int ld = 0;
  const float* const* in_tab = nullptr;
  float* const* out_tab = nullptr;
};

cudaError_t eng_prepare();
cudaError_t eng_launch_ir(int log2B, int spec, EngChan* chans, const EngUpd* upd, int nupd, int maxP,
                          const float2* tw, cudaStream_t st);
// IR spectra of the levels of one size class (2^log2N) listed in upd.
cudaError_t eng_launch_level_ir(int log2N, int spec, EngLevel* levels, const EngLvlUpd* upd, int nupd, int maxK,
                                const float2* tw, cudaStream_t st);
// One audio block for every channel slot: nslots head CTAs plus tail_ctas
// persistent CTAs over the work items [0, nitems). `total` is the number of
// CTAs of every kernel of this block (this one and the level heads launched
// beside it): the last of them to finish advances the channel state.
// `tw_stage`: the heads copy the twiddle table into shared memory (a launch
// of few heads) instead of reading it through L1.
cudaError_t eng_launch_block(int log2B, int spec, EngChan* chans, int nslots, const EngItem* items, int nitems,
                             int tail_ctas, const EngLevel* levels, const EngRows& rows, const float2* tw,
                             bool tw_stage, EngSync sync, unsigned total, cudaStream_t st);
// Level heads of one size class (2^log2N) for a block at which that size is
// due: one CTA per level record [0, nlev) of `levels` (the class's table).
cudaError_t eng_launch_level_heads(int log2B, int log2N, int spec, EngChan* chans, int nslots, const EngLevel* levels,
                                   int nlev, const EngRows& rows, const float2* tw, EngSync sync, unsigned total,
                                   cudaStream_t st);
// CTAs eng_launch_block / eng_launch_level_heads start for these arguments.
unsigned eng_block_ctas(int nslots, int tail_ctas);
// Sets `pending` on channel slots [first, first + n) (the values travel as
// kernel parameters, so the host mirror may change as soon as this returns).
cudaError_t eng_launch_mark_pending(EngChan* chans, int first, int n, cudaStream_t st);
// Partial sums of newly committed IRs (channels with pending set) for the
// coming block, over the base-level work items among [item0, item0 + nitems).
cudaError_t eng_launch_commit(int log2B, int spec, const EngChan* chans, const EngItem* items, int item0,
                              int nitems, int grid, const long long* block, cudaStream_t st);
// A newly committed IR's level state for the coming block k: the partial
// sums of the level items among [item0, item0 + nitems) for the level blocks
// whose heads come at or after k (both parities), from the current delay lines.
cudaError_t eng_launch_level_commit_items(int log2B, int spec, const EngChan* chans, const EngLevel* levels,
                                          const EngItem* items, int item0, int nitems, int max_slices, int grid,
                                          const long long* block, cudaStream_t st);
// A newly committed IR's output for the level blocks whose heads have run but
// whose output is still to be played from block k on: recomputed over every
// partition and written into the new IR's ring (records [first, first + n) of
// one size class, up to nfl blocks each).
cudaError_t eng_launch_level_commit_out(int log2B, int log2N, int spec, const EngChan* chans,
                                        const EngLevel* levels, int first, int n, int nfl, const float2* tw,
                                        const long long* block, cudaStream_t st);

}  // namespace tanb
