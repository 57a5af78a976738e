// C++ caller of the TANConvolution-shaped adapter (include/tanb_convolution.hpp),
// written the way tan/tests/src/TALibTestConvolution/TALibTestConvolution.cpp
// drives amf::TANConvolution: create context, create convolution, Init,
// UpdateResponseTD with BLOCK_UNTIL_READY, then Process block by block; halfway
// the stream moves to a second object by Snapshot / Restore.
// Known answer: a delta IR at tap 10 with gain 0.9 (the testresponse.wav
// channel-0 response) delays and scales the input; block 0 is the crossfade
// from the initial zero IR. Exit code 0 on success.
#include <cmath>
#include <cstdio>
#include <vector>

#include "tanb_convolution.hpp"

int main() {
  const uint32_t C = 2, B = 128, L = 32768, nblocks = 64;
  tanb::TANContext ctx;
  if (ctx.Create(TANB_FULL_VERSION, 0) != TANB_OK) {
    std::printf("TANCreateContext failed: %s\n", tanb_last_error());
    return 2;
  }
  tanb::TANConvolution conv;
  if (conv.Create(ctx) != TANB_OK) return 3;
  if (conv.InitGpu(TANB_METHOD_FHT_UNIFORM_PARTITIONED, L, B, C) != TANB_OK) {
    std::printf("Init failed: %s\n", tanb_last_error());
    return 4;
  }
  std::vector<std::vector<float>> ir(C, std::vector<float>(L, 0.f));
  const float gain = 29491.0f / 32768.0f;
  for (uint32_t c = 0; c < C; ++c) ir[c][10] = gain;
  float* irp[2] = {ir[0].data(), ir[1].data()};
  if (conv.UpdateResponseTD(irp, L, nullptr, TANB_OPERATION_FLAG_BLOCK_UNTIL_READY) != TANB_OK) return 5;

  std::vector<std::vector<float>> in(C, std::vector<float>(B * nblocks)), out(C, std::vector<float>(B * nblocks));
  uint32_t seed = 12345;
  for (auto& ch : in)
    for (auto& s : ch) {
      seed = seed * 1664525u + 1013904223u;
      s = (float)((seed >> 8) & 0xFFFF) / 32768.0f - 1.0f;
    }
  uint32_t flags[2] = {0, 0};
  // halfway through, the stream moves to a second object through a snapshot
  tanb::TANConvolution moved;
  if (moved.Create(ctx) != TANB_OK || moved.InitGpu(TANB_METHOD_FHT_UNIFORM_PARTITIONED, L, B, C) != TANB_OK) return 7;
  tanb::TANConvolution* cur = &conv;
  for (uint32_t b = 0; b < nblocks; ++b) {
    if (b == nblocks / 2) {
      std::vector<uint8_t> snap;
      if (conv.Snapshot(snap) != TANB_OK || moved.Restore(snap) != TANB_OK) {
        std::printf("snapshot / restore failed: %s\n", tanb_last_error());
        return 8;
      }
      cur = &moved;
    }
    float* ip[2] = {in[0].data() + b * B, in[1].data() + b * B};
    float* op[2] = {out[0].data() + b * B, out[1].data() + b * B};
    size_t done = 0;
    if (cur->Process(ip, op, B, flags, &done) != TANB_OK || done != B) {
      std::printf("Process failed at block %u: %s\n", b, tanb_last_error());
      return 6;
    }
  }
  double maxerr = 0.0;
  for (uint32_t c = 0; c < C; ++c)
    for (uint32_t n = 10; n < B * nblocks; ++n) {
      double w = n < B ? (double)n / B : 1.0;
      double e = std::fabs(out[c][n] - w * gain * in[c][n - 10]);
      if (e > maxerr) maxerr = e;
    }
  std::printf("adapter known-answer max error %.3e\n", maxerr);
  conv.Release();
  moved.Release();
  ctx.Release();
  return maxerr < 2e-6 ? 0 : 1;
}
