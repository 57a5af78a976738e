// tanb_convolution.hpp -- C++ TANConvolution-shaped adapter over include/tanb.h.
//
// The method set and argument meaning follow amf::TANConvolution
// (tan/tanlibrary/include/TrueAudioNext.h:125-253), with AMF_RESULT codes as
// int32_t and the cl_mem overloads taking CUDA device pointers. Only the AMF
// values the boundary needs are re-declared (no AMF or OpenCL headers).
// Header-only; link against libtanb.so.
#pragma once

#include <cstddef>
#include <cstdint>

#include <vector>

#include "tanb.h"

namespace tanb {

using AMF_RESULT = int32_t;

// TANCreateContext / TANContext (TrueAudioNext.h:580-597, 647).
class TANContext {
 public:
  TANContext() = default;
  TANContext(const TANContext&) = delete;
  TANContext& operator=(const TANContext&) = delete;
  ~TANContext() { Release(); }

  // TANCreateContext(TAN_FULL_VERSION, &ctx); `device` selects the CUDA device
  // (the reference's InitOpenCL queues).
  AMF_RESULT Create(uint64_t version = TANB_FULL_VERSION, int32_t device = 0) {
    Release();
    return tanb_create_context(version, device, &ctx_);
  }
  void Release() {
    if (ctx_) tanb_context_release(ctx_);
    ctx_ = nullptr;
  }
  tanb_context* get() const { return ctx_; }

 private:
  tanb_context* ctx_ = nullptr;
};

// TANCreateConvolution / TANConvolution (TrueAudioNext.h:125-253, 650-652).
class TANConvolution {
 public:
  TANConvolution() = default;
  TANConvolution(const TANConvolution&) = delete;
  TANConvolution& operator=(const TANConvolution&) = delete;
  ~TANConvolution() { Release(); }

  AMF_RESULT Create(TANContext& ctx) {
    Release();
    return tanb_create_convolution(ctx.get(), &conv_);
  }
  void Release() {
    if (conv_) tanb_convolution_release(conv_);
    conv_ = nullptr;
  }

  AMF_RESULT Init(uint32_t method, uint32_t responseLengthInSamples, uint32_t bufferSizeInSamples,
                  uint32_t channels) {
    return tanb_convolution_init(conv_, method, responseLengthInSamples, bufferSizeInSamples, channels);
  }
  AMF_RESULT InitCpu(uint32_t m, uint32_t l, uint32_t b, uint32_t c) { return Init(m, l, b, c); }
  AMF_RESULT InitGpu(uint32_t m, uint32_t l, uint32_t b, uint32_t c) { return Init(m, l, b, c); }
  AMF_RESULT Terminate() { return tanb_convolution_terminate(conv_); }

  AMF_RESULT UpdateResponseTD(float* ppBuffer[], size_t numOfSamplesToProcess, const uint32_t flagMasks[],
                              const uint32_t operationFlags) {
    return tanb_convolution_update_response_td(conv_, ppBuffer, numOfSamplesToProcess, flagMasks, operationFlags);
  }
  // cl_mem overload -> device pointers
  AMF_RESULT UpdateResponseTDDevice(float* ppDeviceBuffer[], size_t numOfSamplesToProcess,
                                    const uint32_t flagMasks[], const uint32_t operationFlags) {
    return tanb_convolution_update_response_td_device(conv_, ppDeviceBuffer, numOfSamplesToProcess, flagMasks,
                                                      operationFlags);
  }
  AMF_RESULT UpdateResponseFD(float* ppBuffer[], size_t numOfSamplesToProcess, const uint32_t flagMasks[],
                              const uint32_t operationFlags) {
    return tanb_convolution_update_response_fd(conv_, ppBuffer, numOfSamplesToProcess, flagMasks, operationFlags);
  }

  AMF_RESULT Process(float* ppBufferInput[], float* ppBufferOutput[], size_t numOfSamplesToProcess,
                     const uint32_t flagMasks[], size_t* pNumOfSamplesProcessed) {
    return tanb_convolution_process(conv_, ppBufferInput, ppBufferOutput, numOfSamplesToProcess, flagMasks,
                                    pNumOfSamplesProcessed);
  }
  // Process(float* in[], cl_mem out[]) -> device output pointers
  AMF_RESULT ProcessHostToDevice(float* ppBufferInput[], float* ppDeviceOutput[], size_t numOfSamplesToProcess,
                                 const uint32_t flagMasks[], size_t* pNumOfSamplesProcessed) {
    return tanb_convolution_process_host_to_device(conv_, ppBufferInput, ppDeviceOutput, numOfSamplesToProcess,
                                                   flagMasks, pNumOfSamplesProcessed);
  }
  // Process(cl_mem in[], cl_mem out[]) -> device pointers, asynchronous
  AMF_RESULT ProcessDevice(float* ppDeviceInput[], float* ppDeviceOutput[], size_t numOfSamplesToProcess,
                           const uint32_t flagMasks[], size_t* pNumOfSamplesProcessed) {
    return tanb_convolution_process_device(conv_, ppDeviceInput, ppDeviceOutput, numOfSamplesToProcess, flagMasks,
                                           pNumOfSamplesProcessed);
  }
  AMF_RESULT ProcessDirect(float* ppImpulseResponse[], float* ppBufferInput[], float* ppBufferOutput[],
                           size_t numOfSamplesToProcess, size_t* pNumOfSamplesProcessed,
                           int* nzFirstLast = nullptr) {
    return tanb_convolution_process_direct(conv_, ppImpulseResponse, ppBufferInput, ppBufferOutput,
                                           numOfSamplesToProcess, pNumOfSamplesProcessed, nzFirstLast);
  }
  AMF_RESULT ProcessFinalize() { return tanb_convolution_process_finalize(conv_); }
  AMF_RESULT GetNextFreeChannel(uint32_t* pChannelIndex, const uint32_t flagMasks[]) {
    return tanb_convolution_get_next_free_channel(conv_, pChannelIndex, flagMasks);
  }

  // No reference counterpart.
  AMF_RESULT Synchronize() { return tanb_convolution_synchronize(conv_); }
  // The stream state to and from host memory (checkpoint, or a move to an
  // object with the same Init on another GPU).
  AMF_RESULT Snapshot(std::vector<uint8_t>& out) {
    uint64_t n = 0;
    AMF_RESULT r = tanb_convolution_snapshot_bytes(conv_, &n);
    if (r != TANB_OK) return r;
    out.resize((size_t)n);
    return tanb_convolution_snapshot(conv_, out.data(), n);
  }
  AMF_RESULT Restore(const std::vector<uint8_t>& in) { return tanb_convolution_restore(conv_, in.data(), in.size()); }
  tanb_convolution* get() const { return conv_; }

 private:
  tanb_convolution* conv_ = nullptr;
};

}  // namespace tanb
