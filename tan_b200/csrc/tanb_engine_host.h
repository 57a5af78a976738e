// Internal host interface of the batched engine for the drop-in object's
// non-uniform methods (tanb_convolution.cpp runs them on a private engine with
// one session). Not part of the public ABI.
#pragma once

#include <stdint.h>

#include "../../include/tanb.h"
#include "tanb_engine.h"

namespace tanb {

// UpdateResponseTD for the session's channels with mask[j] != 0 (all when
// mask is null); the others keep their IR.
int32_t engine_update_channels(tanb_engine* e, int32_t session, const float* const* ir, size_t n, bool device,
                               uint32_t op, const uint8_t* mask);
// Clears channel `channel` of the session: delay lines, history, partial sums,
// level rings (the IR spectra stay), on the audio stream.
int32_t engine_flush_channel(tanb_engine* e, int32_t session, int channel);
// Arena bytes a non-uniform session of this shape takes in an engine of
// `block` and `spectrum` (0 when the schedule is invalid).
size_t engine_nu_session_bytes(int block, int spectrum, int channels, uint32_t ir_length, uint32_t nlevels,
                               const uint32_t* level_block, const uint32_t* level_parts);
// One block with the given rows (direct launches on the audio stream).
int32_t engine_process_rows(tanb_engine* e, const EngRows& rows);

}  // namespace tanb
