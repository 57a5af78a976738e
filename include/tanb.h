/*
 * tanb.h -- C ABI of the B200-native TrueAudio Next convolution path.
 *
 * Every entry point here stands in for one member of amf::TANConvolution or one
 * TAN factory function (tan/tanlibrary/include/TrueAudioNext.h); the comment
 * above each names the reference declaration it replaces. Arguments keep the
 * reference's meaning; C++ references and cl_mem become plain pointers (device
 * pointers where the reference takes cl_mem). Return values are AMF_RESULT
 * codes (amf/public/include/core/Result.h:43-125).
 *
 * Threading: one tanb_convolution is driven by one thread at a time for
 * Process* and by one thread at a time for UpdateResponse*, like the
 * reference's per-object locks (ConvolutionImpl.h:210-216). Each object owns a
 * CUDA stream on its context's device.
 */
#ifndef TANB_H
#define TANB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* AMF_RESULT subset (amf/public/include/core/Result.h:43-125). */
enum {
  TANB_OK = 0,
  TANB_FAIL = 1,
  TANB_UNEXPECTED = 2,
  TANB_INVALID_ARG = 4,
  TANB_OUT_OF_RANGE = 5,
  TANB_OUT_OF_MEMORY = 6,
  TANB_INVALID_POINTER = 7,
  TANB_NOT_IMPLEMENTED = 9,
  TANB_NOT_SUPPORTED = 10,
  TANB_NOT_FOUND = 11,
  TANB_ALREADY_INITIALIZED = 12,
  TANB_NOT_INITIALIZED = 13,
  TANB_WRONG_STATE = 15,
  TANB_NO_DEVICE = 17,
  TANB_TAN_CLIPPING_WAS_REQUIRED = 42,
  TANB_TAN_UNSUPPORTED_VERSION = 43
};

/* TAN_CONVOLUTION_METHOD (TrueAudioNext.h:81-99). */
enum {
  TANB_METHOD_FFT_OVERLAP_ADD = 0,
  TANB_METHOD_FFT_PARTITIONED_UNIFORM = 1,
  TANB_METHOD_FFT_PARTITIONED_NONUNIFORM = 2,
  TANB_METHOD_FFT_UNIFORM_PARTITIONED = 3,
  TANB_METHOD_FHT_UNIFORM_PARTITIONED = 4,
  TANB_METHOD_FFT_UNIFORM_HEAD_TAIL = 5,
  TANB_METHOD_FHT_UNIFORM_HEAD_TAIL = 6,
  TANB_METHOD_TIME_DOMAIN = 7,
  TANB_METHOD_FHT_NONUNIFORM_PARTITIONED = 8,
  TANB_METHOD_FFT_NONUNIFORM_PARTITIONED = 9,
  TANB_METHOD_USE_PROCESS_FINALIZE = 0x8000,
  TANB_METHOD_USE_PROCESS_TAILTHREAD = 0xC000
};

/* TAN_CONVOLUTION_CHANNEL_FLAG (TrueAudioNext.h:105-110). */
enum {
  TANB_CHANNEL_FLAG_PROCESS = 0,
  TANB_CHANNEL_FLAG_STOP_INPUT = 0x01,
  TANB_CHANNEL_FLAG_FLUSH_STREAM = 0x02
};

/* TAN_CONVOLUTION_OPERATION_FLAG (TrueAudioNext.h:116-120). */
enum {
  TANB_OPERATION_FLAG_NONE = 0x00,
  TANB_OPERATION_FLAG_BLOCK_UNTIL_READY = 0x01
};

/* TAN_FULL_VERSION layout (TrueAudioNext.h:43-52): major in bits 48..63. */
#define TANB_VERSION_MAJOR 1
#define TANB_VERSION_MINOR 3
#define TANB_FULL_VERSION                                          \
  (((uint64_t)TANB_VERSION_MAJOR << 48) | ((uint64_t)TANB_VERSION_MINOR << 32) | \
   ((uint64_t)1 << 16) | (uint64_t)1)

typedef struct tanb_context tanb_context;
typedef struct tanb_convolution tanb_convolution;

/* TANCreateContext(amf_uint64 version, TANContext**) -- TrueAudioNext.h:647,
 * TANContextImpl.cpp:87-127. Major version must be 1. `device` is the CUDA
 * device ordinal the context's objects run on (the reference's OpenCL
 * queues, TANContext::InitOpenCL, TrueAudioNext.h:587-592). */
int32_t tanb_create_context(uint64_t version, int32_t device, tanb_context** ctx);

/* TANContext::Release (AMFInterface refcount, amf/public/include/core/Interface.h:63-80). */
int32_t tanb_context_release(tanb_context* ctx);

/* TANCreateConvolution(TANContext*, TANConvolution**) -- TrueAudioNext.h:650-652,
 * ConvolutionImpl.cpp:66-80. */
int32_t tanb_create_convolution(tanb_context* ctx, tanb_convolution** conv);

/* TANConvolution::Release (Interface.h:63-80); also terminates. */
int32_t tanb_convolution_release(tanb_convolution* conv);

/* TANConvolution::Init / InitCpu / InitGpu (TrueAudioNext.h:134-146,
 * ConvolutionImpl.cpp:179-281, 1113-1259). `method` is a TANB_METHOD_* value,
 * optionally or-ed with TANB_METHOD_USE_PROCESS_FINALIZE. The uniform
 * partitioned and head/tail methods run the uniformly-partitioned path; the
 * non-uniform methods (TANB_METHOD_FFT_PARTITIONED_NONUNIFORM,
 * _FHT_NONUNIFORM_PARTITIONED, _FFT_NONUNIFORM_PARTITIONED) run levels of
 * growing block size along the IR (see tanb_convolution_init_nu); bufferSize
 * must be a power of two in [32, 8192] (the reference's GPU rule, :1136-1146). */
int32_t tanb_convolution_init(tanb_convolution* conv, uint32_t method,
                              uint32_t responseLengthInSamples,
                              uint32_t bufferSizeInSamples, uint32_t channels);

/* No reference counterpart: Init of a non-uniform method
 * (TANB_METHOD_FFT_PARTITIONED_NONUNIFORM, _FHT_NONUNIFORM_PARTITIONED or
 * _FFT_NONUNIFORM_PARTITIONED) with an explicit level schedule, as
 * tanb_engine_open_session_nu takes it (level_block[0] = bufferSize), for a
 * schedule chosen by the autotuner. tanb_convolution_init picks a default
 * schedule for those methods: two partitions per size doubling from the block
 * to about L / 32 (at most 16384), the largest size taking the rest. The
 * non-uniform methods run blocks in [128, 2048] (else AMF_NOT_SUPPORTED); an IR
 * update takes effect on the next block, even for a channel that is free at
 * the time (the uniform methods apply it at the channel's next running block). */
int32_t tanb_convolution_init_nu(tanb_convolution* conv, uint32_t method, uint32_t responseLengthInSamples,
                                 uint32_t bufferSizeInSamples, uint32_t channels, uint32_t nlevels,
                                 const uint32_t* level_block, const uint32_t* level_parts);

/* TANConvolution::Terminate (TrueAudioNext.h:148, ConvolutionImpl.cpp:307-352). */
int32_t tanb_convolution_terminate(tanb_convolution* conv);

/* TANConvolution::UpdateResponseTD(float* ppBuffer[], ...) -- TrueAudioNext.h:158-162,
 * ConvolutionImpl.cpp:357-382, 407-695. Host IRs, one array per channel of
 * numOfSamples <= responseLength floats. Channels flagged STOP_INPUT keep
 * their IR; FLUSH_STREAM channels are flushed. The new IR takes effect, with
 * a one-block linear crossfade, on the next processed block. The caller may
 * reuse the IR buffers as soon as this returns. */
int32_t tanb_convolution_update_response_td(tanb_convolution* conv,
                                            const float* const* ppBuffer,
                                            size_t numOfSamples,
                                            const uint32_t* flagMasks,
                                            uint32_t operationFlags);

/* TANConvolution::UpdateResponseTD(cl_mem ppBuffer[], ...) -- TrueAudioNext.h:163-167.
 * Same as above with device-resident IR arrays. */
int32_t tanb_convolution_update_response_td_device(tanb_convolution* conv,
                                                   const float* const* ppDeviceBuffer,
                                                   size_t numOfSamples,
                                                   const uint32_t* flagMasks,
                                                   uint32_t operationFlags);

/* TANConvolution::UpdateResponseFD (both overloads) -- TrueAudioNext.h:177-186,
 * ConvolutionImpl.cpp:697-717: not supported, as in the reference. */
int32_t tanb_convolution_update_response_fd(tanb_convolution* conv,
                                            const float* const* ppBuffer,
                                            size_t numOfSamples,
                                            const uint32_t* flagMasks,
                                            uint32_t operationFlags);

/* TANConvolution::Process(float* in[], float* out[], ...) -- TrueAudioNext.h:200-205,
 * ConvolutionImpl.cpp:809-1043. Host buffers. Processes every whole block of
 * bufferSize samples in numOfSamples; *pNumOfSamplesProcessed (nullable) gets
 * that count. Outputs of stopped (free) channels are left untouched. */
int32_t tanb_convolution_process(tanb_convolution* conv,
                                 const float* const* ppBufferInput,
                                 float* const* ppBufferOutput,
                                 size_t numOfSamples,
                                 const uint32_t* flagMasks,
                                 size_t* pNumOfSamplesProcessed);

/* TANConvolution::Process(float* in[], cl_mem out[], ...) -- TrueAudioNext.h:207-212,
 * ConvolutionImpl.cpp:782-806. Host input, device output arrays. */
int32_t tanb_convolution_process_host_to_device(tanb_convolution* conv,
                                                const float* const* ppBufferInput,
                                                float* const* ppDeviceOutput,
                                                size_t numOfSamples,
                                                const uint32_t* flagMasks,
                                                size_t* pNumOfSamplesProcessed);

/* TANConvolution::Process(cl_mem in[], cl_mem out[], ...) -- TrueAudioNext.h:215-220
 * (AMF_NOT_IMPLEMENTED in the reference, ConvolutionImpl.cpp:835-845; implemented
 * here). Device input and output arrays; returns once the work is enqueued on
 * the object's stream (see tanb_convolution_synchronize). */
int32_t tanb_convolution_process_device(tanb_convolution* conv,
                                        const float* const* ppDeviceInput,
                                        float* const* ppDeviceOutput,
                                        size_t numOfSamples,
                                        const uint32_t* flagMasks,
                                        size_t* pNumOfSamplesProcessed);

/* Fused PCM pipeline (no single reference counterpart): the per-block chain
 * of samples/src/common/SimpleVRaudio.cpp:1059-1117 -- TANConverter
 * short->float of each channel's input, TANConvolution::Process, TANMixer::Mix
 * of the channels of each output group, TANConverter float->short of each mix
 * -- in one call, the conversions and the mix done inside the head kernel.
 * Channel c reads in[c][i * in_step] (int16, converted as
 * tanb_converter_short_to_float with in_gain) and is mixed into output group
 * group[c] < ngroups <= channels (every group needs a channel); a group sums
 * its channels from 0 in ascending channel order (Mixer.cl:26-41) and its
 * sample i goes to out[g][i * out_step], converted with out_gain by the device
 * float->short rule (Converter.cl:97-120); *clipped reports any clamped
 * sample. Whole blocks of n as tanb_convolution_process; no channel flags;
 * not for TIME_DOMAIN. */
int32_t tanb_convolution_process_mix_pcm16(tanb_convolution* conv, const int16_t* const* in, size_t in_step,
                                           float in_gain, const uint32_t* group, uint32_t ngroups,
                                           int16_t* const* out, size_t out_step, float out_gain, size_t n,
                                           int32_t* clipped, size_t* done);

/* TANConvolution::ProcessDirect(float* ir[], float* in[], float* out[], ...) --
 * TrueAudioNext.h:223-230, ConvolutionImpl.cpp:721-762. TIME_DOMAIN method only
 * (AMF_NOT_SUPPORTED otherwise): direct FIR with a per-call IR over a circular
 * history of nextpow2(responseLength) samples; nzFirstLast (nullable) holds
 * [first, last) nonzero tap bounds per channel. */
int32_t tanb_convolution_process_direct(tanb_convolution* conv,
                                        const float* const* ppImpulseResponse,
                                        const float* const* ppBufferInput,
                                        float* const* ppBufferOutput,
                                        size_t numOfSamples,
                                        size_t* pNumOfSamplesProcessed,
                                        const int32_t* nzFirstLast);

/* TANConvolution::ProcessFinalize -- TrueAudioNext.h:232, ConvolutionImpl.cpp:1046-1079.
 * With TANB_METHOD_USE_PROCESS_FINALIZE, Process returns after the head
 * (partition 0) and this call enqueues the tail for the next block. */
int32_t tanb_convolution_process_finalize(tanb_convolution* conv);

/* TANConvolution::GetNextFreeChannel -- TrueAudioNext.h:247-249,
 * ConvolutionImpl.cpp:1084-1110. */
int32_t tanb_convolution_get_next_free_channel(tanb_convolution* conv,
                                               uint32_t* pChannelIndex,
                                               const uint32_t* flagMasks);

/* No reference counterpart (the reference's CPU path is synchronous): waits
 * until all work enqueued by this object has finished. */
int32_t tanb_convolution_synchronize(tanb_convolution* conv);

/* No reference counterpart: the object's CUDA stream (a cudaStream_t), for
 * callers that order their own device work after Process_device. */
void* tanb_convolution_stream(tanb_convolution* conv);

/* No reference counterpart: layout facts for tools and tests --
 * out[0] = partitions P, out[1] = block B, out[2] = channels C,
 * out[3] = device bytes held by the object. */
int32_t tanb_convolution_info(tanb_convolution* conv, int64_t out[4]);

/* No reference counterpart: autotuner hook. index >= 0 selects entry `index`
 * of the tail kernel's compiled tilings (TANB_OUT_OF_RANGE past the last);
 * index < 0 only reads. out (nullable) gets the tiling in use: units of two
 * bins per CTA row, partition splits per CTA, partitions in flight per thread. */
int32_t tanb_convolution_tiling(tanb_convolution* conv, int32_t index, int32_t out[3]);

/* No reference counterpart: per-kernel device-time accounting. With enable
 * != 0 every kernel this object launches is bracketed by a CUDA event pair on
 * its stream. */
int32_t tanb_convolution_profile(tanb_convolution* conv, int32_t enable);

/* No reference counterpart: reads and resets the accounting --
 * counts[0..2] = launches of the head, tail and IR-spectrum kernels since the
 * last read, counts[3..5] = how many of those were timed, ms[0..2] = their
 * summed device milliseconds. Waits for the timed launches to finish. */
int32_t tanb_convolution_profile_read(tanb_convolution* conv, int64_t counts[6], double ms[3]);

/* No reference counterpart (checkpoint / migration): a snapshot of the object's
 * stream state -- both IR slots' spectra, the delay line, the overlap-save
 * history, the tail rows (a pending IR's too), the delay-line position, the
 * block count and the per-channel swap and flag state -- in a caller buffer
 * of tanb_convolution_snapshot_bytes bytes (host memory, pageable or not).
 * tanb_convolution_restore loads one into an object with the same Init
 * (method, IR length, block, channels), on this GPU or another: its stream
 * then continues with the same output, bit for bit. Snapshot runs a tail that
 * finalize mode deferred and waits for the object's stream; restore discards
 * the target's own state. Uniformly partitioned methods only
 * (TANB_NOT_SUPPORTED for TIME_DOMAIN and the non-uniform methods);
 * TANB_INVALID_ARG for a short buffer or a snapshot of another configuration. */
int32_t tanb_convolution_snapshot_bytes(tanb_convolution* conv, uint64_t* bytes);
int32_t tanb_convolution_snapshot(tanb_convolution* conv, void* buffer, uint64_t bytes);
int32_t tanb_convolution_restore(tanb_convolution* conv, const void* buffer, uint64_t bytes);

/* No reference counterpart: host microseconds of the last Process call of the
 * uniformly partitioned methods, by part -- us[0] staging the rows and
 * descriptors, us[1] launching the kernels, us[2] waiting for the heads'
 * completion signal (host outputs only), us[3] copying the outputs to the
 * caller's rows, us[4] the whole call -- and us[5] which caller rows the
 * kernels read or wrote in place (1: inputs, 2: outputs; host rows that sit
 * at one stride in one page-locked allocation are not staged). */
int32_t tanb_convolution_call_times(tanb_convolution* conv, double us[6]);

/* No reference counterpart; a test hook for failure handling. Sets how many
 * times the tail kernel's cp.async.bulk pipelines poll a stage's barrier
 * before giving up (default and maximum 2^20; negative: the default). On a
 * timeout the kernel records the error, waits with the full bound for its
 * copies in flight and exits; Process or Synchronize then return AMF_FAIL.
 * A bound of 0 makes the first wait give up at once, so that the failure
 * path runs without any fault. */
int32_t tanb_convolution_set_wait_limit(tanb_convolution* conv, int32_t polls);

/* ---------------------------------------------------------------------------
 * Batched engine. No single reference counterpart: it is the serving form of
 * the same path -- many TANConvolution-equivalent sessions (C channels, IR
 * length L each) processed together in ONE kernel launch per audio block (heads
 * of every channel side by side with the partition multiply-accumulate work
 * items for the next block), the role the reference's GPU engine plays with
 * its channel maps (tan/tanlibrary/src/Graal/GraalConv.cpp:644-704, 1883-2145).
 * ------------------------------------------------------------------------- */
typedef struct tanb_engine tanb_engine;

enum { TANB_SPECTRUM_FP32 = 0, TANB_SPECTRUM_FP16 = 1, TANB_SPECTRUM_BF16 = 2, TANB_SPECTRUM_FP24 = 3 };

/* Creates an engine for blocks of `block` samples (power of two in
 * [128, 2048]). IR spectra are stored as `spectrum`: FP16 / BF16 with a
 * power-of-two scale per partition, or FP24 (engine only: FP32 rounded to a
 * 15-bit fraction, 6 bytes per complex bin) for the IR spectra AND the input
 * delay line, a quarter fewer streamed bytes than FP32 at an output error near
 * -100 dB; accumulation is FP32 in every case. Sessions are
 * admitted while their device memory fits in `budget_bytes`; at most
 * `max_channels` channel slots. `partitions_per_item` (0: 32) sets the size of
 * the tail's work items. */
int32_t tanb_engine_create(tanb_context* ctx, uint32_t block, uint32_t spectrum, uint64_t budget_bytes,
                           uint32_t max_channels, uint32_t partitions_per_item, tanb_engine** engine);
int32_t tanb_engine_release(tanb_engine* engine);

/* Admits a session of `channels` channels and IR length `ir_length`; its
 * channels occupy slots [*first_slot, *first_slot + channels) of the I/O
 * buffers. AMF_OUT_OF_MEMORY when the budget or the slot table is exhausted.
 * The session starts with an all-zero IR. */
int32_t tanb_engine_open_session(tanb_engine* engine, uint32_t channels, uint32_t ir_length, int32_t* session,
                                 uint32_t* first_slot);
/* Admits a non-uniformly partitioned session (the reference's
 * TAN_CONVOLUTION_METHOD_*_NONUNIFORM methods, ConvolutionImpl.cpp:224-246,
 * 2416-2428): level 0 has the engine's block and level_parts[0] partitions;
 * level l >= 1 has block level_block[l] (a power of two above level l-1's, at
 * most 16384) and level_parts[l] partitions starting at tap
 * o_l = sum_{m<l} level_block[m] * level_parts[m], which must be >= its block
 * (no added latency); the levels must cover ir_length. Every level runs in the
 * same graph launch per block as every other session: its tail spread over
 * the blocks of its period, its head beside the block launch at the blocks
 * where its block completes. IR updates crossfade over one block exactly as
 * for a uniform session (the new IR's output of the level blocks already
 * computed is recomputed when the update is committed). */
int32_t tanb_engine_open_session_nu(tanb_engine* engine, uint32_t channels, uint32_t ir_length, uint32_t nlevels,
                                    const uint32_t* level_block, const uint32_t* level_parts, int32_t* session,
                                    uint32_t* first_slot);
int32_t tanb_engine_close_session(tanb_engine* engine, int32_t session);

/* Device bytes a session of this shape takes from the budget of an engine
 * created with `block`, `spectrum` and `partitions_per_item` (0: 32):
 * nlevels = 0 for a uniformly partitioned session, else the level schedule of
 * tanb_engine_open_session_nu. Host arithmetic only (no device needed), so a
 * router can place sessions on GPUs by the engines' own admission rule. */
int32_t tanb_engine_session_bytes(uint32_t block, uint32_t spectrum, uint32_t partitions_per_item, uint32_t channels,
                                  uint32_t ir_length, uint32_t nlevels, const uint32_t* level_block,
                                  const uint32_t* level_parts, uint64_t* bytes);

/* UpdateResponseTD for one session (host IR rows, n <= ir_length). The IR is
 * copied before this returns and transformed on the engine's update stream,
 * off the audio path; it takes effect, with a one-block crossfade, on the
 * first tanb_engine_process* call after the transform has finished. With
 * TANB_OPERATION_FLAG_BLOCK_UNTIL_READY the call waits for the transform, so
 * the swap lands on the next block (the reference flag's meaning,
 * TrueAudioNext.h:112-120). May be called from another thread than Process. */
int32_t tanb_engine_update_response_td(tanb_engine* engine, int32_t session, const float* const* ir, size_t n,
                                       uint32_t operationFlags);
/* Same with device-resident IR rows. */
int32_t tanb_engine_update_response_td_device(tanb_engine* engine, int32_t session, const float* const* ir,
                                              size_t n, uint32_t operationFlags);

/* Pinned host I/O buffers [max_channels][block]: write slot s's input block at
 * in[s * block], read its output at out[s * block] after tanb_engine_process.
 * The block launch reads and writes them in place (mapped host memory). */
int32_t tanb_engine_io(tanb_engine* engine, float** in, float** out);

/* Copies `count` input rows of `block` samples, row j from src + j * ld, into
 * the pinned input buffer at slots [first_slot, first_slot + count), spread
 * over host threads for large copies. Call between tanb_engine_process calls
 * (the block launch reads the buffer in place). */
int32_t tanb_engine_write_input(tanb_engine* engine, uint32_t first_slot, const float* src, uint32_t count,
                                size_t ld);

/* One block for every open session through the host buffers (one CUDA graph
 * holding the block launch); returns when the output is in the pinned output
 * buffer. */
int32_t tanb_engine_process(tanb_engine* engine);

/* One block with device-resident I/O: slot s reads in[s * ld] (null: silence)
 * and writes out[s * ld]. Asynchronous on the engine's stream. */
int32_t tanb_engine_process_device(tanb_engine* engine, const float* in, float* out, uint32_t ld);

int32_t tanb_engine_synchronize(tanb_engine* engine);
void* tanb_engine_stream(tanb_engine* engine);

/* out[0] sessions, out[1] channels, out[2] slot high-water mark, out[3] work
 * items high-water mark, out[4] arena bytes in use, out[5] budget, out[6]
 * algorithmic bytes of one block launch (heads and work items), out[7] tail
 * CTAs of the block launch at most. */
int32_t tanb_engine_info(tanb_engine* engine, int64_t out[8]);

/* No reference counterpart (checkpoint / migration of a session): a snapshot
 * of a uniformly partitioned session -- both IR slots' spectra (and scales),
 * delay lines, input history, partial-sum rows, each channel's delay-line
 * position and IR slot, the session's block count and an IR update staged but
 * not yet in effect -- in a caller buffer of
 * tanb_engine_session_snapshot_bytes bytes (host memory). The snapshot waits
 * for the engine's streams. tanb_engine_open_session_restore opens a session
 * from one in an engine with the same block, spectrum and partitions per item
 * (on this GPU or another) whose output continues bit for bit from the next
 * block on. TANB_NOT_SUPPORTED for non-uniform sessions; TANB_INVALID_ARG for
 * a short buffer or a snapshot of another engine configuration; admission as
 * for tanb_engine_open_session. */
int32_t tanb_engine_session_snapshot_bytes(tanb_engine* engine, int32_t session, uint64_t* bytes);
int32_t tanb_engine_session_snapshot(tanb_engine* engine, int32_t session, void* buffer, uint64_t bytes);
int32_t tanb_engine_open_session_restore(tanb_engine* engine, const void* buffer, uint64_t bytes, int32_t* session,
                                         uint32_t* first_slot);

/* out[0] blocks the session has processed, out[1] its block index at which the
 * last IR update took effect (-1: none yet), out[2] 1 while an update is
 * uploaded but not yet in effect. */
int32_t tanb_engine_session_state(tanb_engine* engine, int32_t session, int64_t out[3]);

/* Accounting: counts[0] block launches, counts[1] commit launches (partial
 * sums of a newly committed IR), counts[2] IR updates, counts[3] blocks timed;
 * ms[0] device milliseconds of the timed block launches (tanb_engine_process_device
 * with profiling enabled), ms[1] 0. Reading resets. */
int32_t tanb_engine_profile(tanb_engine* engine, int32_t enable);
int32_t tanb_engine_profile_read(tanb_engine* engine, int64_t counts[4], double ms[2]);

/* Host-side microseconds of the last tanb_engine_process: us[0] waiting for
 * the engine's lock, us[1] committing staged IR updates, us[2] capturing and
 * instantiating block graphs (0 unless the session tables' shape changed),
 * us[3] launching the block graph, us[4] waiting for the block's outputs,
 * us[5] the whole call; us[6] the longest call since the previous read, us[7]
 * block graphs built since the engine was created. No reference counterpart:
 * serving diagnostics for the real-time block deadline. */
int32_t tanb_engine_block_times(tanb_engine* engine, double us[8]);

/* ---------------------------------------------------------------------------
 * TANConverter (TrueAudioNext.h:344-398; TANCreateConverter :653-656) and
 * TANMixer (TrueAudioNext.h:611-634; TANCreateMixer :657-660), the conversion
 * and mixing steps either side of the convolution. Host-pointer overloads give
 * the reference's CPU results bit for bit (ConverterImpl.cpp:217-408,
 * MixerImpl.cpp:226-250); device-pointer overloads those of its OpenCL kernels
 * (Converter.cl:27-120, Mixer.cl:26-41). All computation runs on the GPU.
 * ------------------------------------------------------------------------- */
enum { TANB_SAMPLE_TYPE_FLOAT = 0, TANB_SAMPLE_TYPE_SHORT = 1 }; /* TrueAudioNext.h:73-77 */

typedef struct tanb_converter tanb_converter;
/* TANCreateConverter + Init / Terminate. */
int32_t tanb_converter_create(tanb_context* ctx, tanb_converter** converter);
int32_t tanb_converter_release(tanb_converter* converter);
/* Convert(short*, inputStep, n, float*, outputStep, gain) (TrueAudioNext.h:353-356):
 * out[i * out_step] = in[i * in_step] * (gain / 32767). */
int32_t tanb_converter_short_to_float(tanb_converter* converter, const int16_t* in, size_t in_step, size_t n,
                                      float* out, size_t out_step, float gain);
/* Convert(float*, inputStep, n, short*, outputStep, gain, bool* clipped)
 * (TrueAudioNext.h:357-360); *clipped (if not null) as the reference reports it. */
int32_t tanb_converter_float_to_short(tanb_converter* converter, const float* in, size_t in_step, size_t n,
                                      int16_t* out, size_t out_step, float gain, int32_t* clipped);
/* Batch forms over `count` buffers (TrueAudioNext.h:363-373). */
int32_t tanb_converter_short_to_float_batch(tanb_converter* converter, const int16_t* const* in, size_t in_step,
                                            size_t n, float* const* out, size_t out_step, float gain,
                                            int32_t count);
int32_t tanb_converter_float_to_short_batch(tanb_converter* converter, const float* const* in, size_t in_step,
                                            size_t n, int16_t* const* out, size_t out_step, float gain,
                                            int32_t count, int32_t* clipped);
/* Device buffers (the cl_mem overloads, TrueAudioNext.h:375-397): buffer i's
 * sample j at in[i] + (in_offsets[i] + j * in_step) elements of in_type, the
 * same for out; offsets may be null (0). Asynchronous on the converter's
 * stream unless `clipped` is requested (then it waits, as the reference). */
int32_t tanb_converter_convert_device(tanb_converter* converter, const void* const* in, size_t in_step,
                                      const size_t* in_offsets, int32_t in_type, void* const* out, size_t out_step,
                                      const size_t* out_offsets, int32_t out_type, size_t n, float gain,
                                      int32_t count, int32_t* clipped);
int32_t tanb_converter_synchronize(tanb_converter* converter);
void* tanb_converter_stream(tanb_converter* converter);

typedef struct tanb_mixer tanb_mixer;
/* TANCreateMixer + Init(buffer_size, num_channels) (TrueAudioNext.h:616). */
int32_t tanb_mixer_create(tanb_context* ctx, size_t buffer_size, int32_t channels, tanb_mixer** mixer);
int32_t tanb_mixer_release(tanb_mixer* mixer);
/* Mix(float* in[], float* out) (TrueAudioNext.h:620-622): host buffers. */
int32_t tanb_mixer_mix(tanb_mixer* mixer, const float* const* in, float* out);
/* Mix(cl_mem in[], cl_mem out) (:625-627) and Mix(cl_mem in, cl_mem out, stride)
 * (:630-633): device buffers, asynchronous on the mixer's stream. */
int32_t tanb_mixer_mix_device(tanb_mixer* mixer, const float* const* in, float* out);
int32_t tanb_mixer_mix_device_strided(tanb_mixer* mixer, const float* in, float* out, size_t input_stride);
int32_t tanb_mixer_synchronize(tanb_mixer* mixer);
void* tanb_mixer_stream(tanb_mixer* mixer);

/* ---------------------------------------------------------------------------
 * GPU-resident IR producer: left / right impulse responses of a shoebox room
 * written into device memory, ready for tanb_convolution_update_response_td_device
 * (the GPU path of TrueAudioVR::generateRoomResponse with GENROOM_USE_GPU_MEM,
 * samples/src/TrueAudioVR/TrueAudioVR.h:153-155, TrueAudioVR.cpp:659-786;
 * kernels Kernels/GenerateRoomResponse.cl:206-321, Kernels/Fill.cl).
 * ------------------------------------------------------------------------- */
typedef struct {                 /* RoomDefinition (TrueAudioVR.h:101-106), meters */
  float width, height, length;
  float damp_left, damp_right, damp_top, damp_bottom, damp_front, damp_back; /* (0, 1] */
} tanb_room;
typedef struct {                 /* MonoSource (TrueAudioVR.h:69-72) */
  float x, y, z;
} tanb_source;
typedef struct {                 /* StereoListener + HeadModel (TrueAudioVR.h:62-81) */
  float head_x, head_y, head_z, ear_spacing;
  float yaw, pitch, roll;        /* degrees */
  int32_t filter_length;         /* <= 64 */
  float low_pass[64], high_pass[64];
} tanb_listener;
enum { TANB_GENROOM_LIMIT_BOUNCES = 0x40 }; /* TrueAudioVR.h:55 */

typedef struct tanb_room_generator tanb_room_generator;
/* Workspace for responses of up to max_length samples. */
int32_t tanb_room_generator_create(tanb_context* ctx, int32_t max_length, tanb_room_generator** generator);
int32_t tanb_room_generator_release(tanb_room_generator* generator);
/* Writes `length` samples of the left and right responses to the device
 * buffers `left` / `right`, asynchronously on `stream` (a cudaStream_t; null:
 * the generator's stream), after any earlier call of this generator. With
 * TANB_GENROOM_LIMIT_BOUNCES at most max_bounces images per axis and side.
 * Results are reproducible bit for bit (exact 64-bit fixed-point sums). */
int32_t tanb_room_response(tanb_room_generator* generator, const tanb_room* room, const tanb_source* source,
                           const tanb_listener* ears, int32_t sample_rate, int32_t length, float* left,
                           float* right, uint32_t flags, int32_t max_bounces, void* stream);
/* Image sources per ear of the last call. */
int64_t tanb_room_images(tanb_room_generator* generator);
int32_t tanb_room_generator_synchronize(tanb_room_generator* generator);
void* tanb_room_generator_stream(tanb_room_generator* generator);

/* ---------------------------------------------------------------------------
 * Non-uniformly partitioned convolution: the TAN_CONVOLUTION_METHOD_*_NONUNIFORM
 * family (CPU variant ConvolutionImpl.cpp:224-246, 2416-2428; GPU two-stream
 * engine tan/tanlibrary/src/Graal2/Reverberate.cpp), with a level schedule of
 * block sizes that grow along the IR. Zero added latency: level l (block N_l,
 * K_l partitions) starts at tap o_l >= N_l, so only the first level is on a
 * block's critical path.
 * ------------------------------------------------------------------------- */
typedef struct tanb_nu tanb_nu;

/* Default schedule: two partitions per size from base_block doubling up to
 * max_block (<= 16384; tanb_nu_create takes blocks up to 8192, engine
 * sessions up to 16384), the largest size covering the rest of the IR.
 * Arrays hold >= 16. */
int32_t tanb_nu_schedule(uint32_t ir_length, uint32_t base_block, uint32_t max_block, uint32_t* nlevels,
                         uint32_t* level_block, uint32_t* level_parts);

/* C channels, IR length, levels (block sizes nondecreasing powers of two in
 * [32, 8192], level 0's block = the base block; each level's first tap >= its
 * block), spectrum TANB_SPECTRUM_*. */
int32_t tanb_nu_create(tanb_context* ctx, uint32_t channels, uint32_t ir_length, uint32_t nlevels,
                       const uint32_t* level_block, const uint32_t* level_parts, uint32_t spectrum, tanb_nu** nu);
int32_t tanb_nu_release(tanb_nu* nu);

/* Host IR rows (n <= ir_length), transformed synchronously; takes effect at the
 * next block without a crossfade (the levels' queued contributions of the old
 * IR still play out). */
int32_t tanb_nu_set_response(tanb_nu* nu, const float* const* ir, size_t n);

/* Pinned host I/O [channels][base_block] and one base block through them. */
int32_t tanb_nu_io(tanb_nu* nu, float** in, float** out);
int32_t tanb_nu_process(tanb_nu* nu);

/* One base block with device I/O, rows of `ld` floats; asynchronous. */
int32_t tanb_nu_process_device(tanb_nu* nu, const float* in, float* out, uint32_t ld);
int32_t tanb_nu_synchronize(tanb_nu* nu);
void* tanb_nu_stream(tanb_nu* nu);

/* out[0] channels, out[1] base block, out[2] levels, out[3] device bytes,
 * out[4] average algorithmic tail bytes per base block, out[5] blocks done. */
int32_t tanb_nu_info(tanb_nu* nu, int64_t out[6]);

/* No reference counterpart. One-shot convolution that allocates no device
 * memory, for callers that cannot call cudaMalloc on this path -- e.g. a
 * plugin inside a host application's real-time audio callback, where an
 * allocation can block for milliseconds, or a host that gives the library a
 * fixed memory budget. out[c * samples + i] = sum_k ir[c * ir_length + k] *
 * in[c * samples + i - k] for every channel c, i < samples (zero history
 * before sample 0); in, ir, out are device arrays, samples a multiple of
 * `block` (power of two in [32, 8192]), work enqueued on `stream`.
 * All temporaries live in one library-owned device array of
 * TANB_NO_ALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit; requests whose working set (about channels * ceil(ir_length / block)
 * * block * 28 bytes plus small per-channel terms) exceeds it return
 * TANB_INVALID_ARG. Calls share that array: calls that overlap on the GPU
 * race, so serialise them. The first call on a device looks up the array's
 * address; make it before any stream capture. */
#define TANB_NO_ALLOC_SCRATCH_BYTES (32u << 20)
int32_t tanb_convolve_no_alloc(const float* in, const float* ir, float* out, uint32_t channels, size_t samples,
                               size_t ir_length, uint32_t block, void* stream);

/* No reference counterpart; a measurement aid. Reads `bytes` of device memory
 * at `src` once (16-byte streaming loads, grid of ctas_per_sm CTAs per SM of
 * `threads` threads) and adds their sum to *out (device float), on `stream`.
 * Timed around one launch, it is the floor a bandwidth-bound launch of that
 * size reaches on this GPU; the bench compares the partition MAC with it. */
int32_t tanb_stream_read(const void* src, size_t bytes, float* out, uint32_t ctas_per_sm, uint32_t threads,
                         void* stream);

/* No reference counterpart: text of the last error raised on this thread. */
const char* tanb_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TANB_H */
