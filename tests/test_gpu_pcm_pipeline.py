"""Fused PCM pipeline (tanb_convolution_process_mix_pcm16) on the GPU, laid out
as the reference's sample pipeline (samples/src/common/SimpleVRaudio.cpp:
1059-1117): S interleaved int16 stereo sources, channel 2*src + ear reads
source src at offset ear with step 2, even channels mix into the left output,
odd into the right, written interleaved (step 2).

Bit for bit it equals the unfused chain: host short->float conversion (the
reference CPU rule), TANConvolution::Process on the GPU, the device mixer rule
and the device float->short rule (restated in the oracle). Against the chain
run wholly on the oracle (CPU convolution) it agrees within 1 LSB."""
import numpy as np
import pytest

from oracle import ref
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _make(ctx, L, B, C):
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    return conv


@pytest.mark.parametrize("S,B,L,out_gain,blocks_per_call", [(3, 256, 3000, 1.0, 1), (8, 512, 9000, 0.5, 3),
                                                            (2, 128, 700, 12.0, 2)])
def test_fused_pipeline_equals_unfused_chain(tan_ctx, S, B, L, out_gain, blocks_per_call):
    g = H.rng(S * 100 + B)
    C, nb = 2 * S, 12
    T = nb * B
    src = [(g.uniform(-0.6, 0.6, 2 * T) * 32767).astype(np.int16) for _ in range(S)]
    h0, h1 = H.irs(g, C, L, (0.5, 1.5)), H.irs(g, C, L, (0.5, 1.5))
    group = np.array([c % 2 for c in range(C)], np.uint32)
    rows_in = [src[c // 2][c % 2:] for c in range(C)]

    fused = _make(tan_ctx, L, B, C)
    pout = np.full(2 * T, 999, np.int16)
    rows_out = [pout[0:], pout[1:]]
    clip_any = False
    k = 0
    while k < nb:
        if k == 0:
            assert fused.UpdateResponseTD(h0, L) == 0
        if k == 6:
            assert fused.UpdateResponseTD(h1, L) == 0
        step = min(blocks_per_call, nb - k, 6 - k if k < 6 else nb - k)
        xs = [r[2 * k * B:] for r in rows_in]
        ys = [r[2 * k * B:] for r in rows_out]
        rc, clip, done = fused.ProcessMixPcm16(xs, 2, 1.0, group, 2, ys, 2, out_gain, step * B)
        assert rc == 0 and done == step * B, cv.last_error()
        clip_any |= clip
        k += step

    # unfused chain, convolution on the GPU
    xf = np.stack([ref.convert_s16_f32(r, 1.0, in_step=2, n=T) for r in rows_in])
    plain = _make(tan_ctx, L, B, C)
    yf, _ = H.run_stream(plain, xf, B, {0: (h0, None), 6: (h1, None)})
    exp, exp_clip = [], False
    for ear in range(2):
        mixed = ref.mix(yf[ear::2], device=True)
        s16, c = ref.convert_f32_s16(mixed, out_gain, device=True)
        exp.append(s16)
        exp_clip |= c
    assert np.array_equal(pout[0::2], exp[0]) and np.array_equal(pout[1::2], exp[1])
    assert clip_any == exp_clip
    if out_gain > 4:
        assert clip_any

    # the whole chain on the oracle: within one LSB
    rc_ = ref.RefConvolution(L, B, C)
    yo, _ = H.run_stream(rc_, xf, B, {0: (h0, None), 6: (h1, None)})
    rc_.close()
    for ear in range(2):
        s16, _ = ref.convert_f32_s16(ref.mix(yo[ear::2], device=True), out_gain, device=True)
        d = np.abs(s16.astype(np.int32) - pout[ear::2].astype(np.int32))
        assert d.max() <= 1 and np.mean(d > 0) < 0.01
    fused.Release()
    plain.Release()


def test_fused_pipeline_errors(tan_ctx):
    B, L, C = 256, 1000, 4
    conv = _make(tan_ctx, L, B, C)
    x = [np.zeros(B, np.int16) for _ in range(C)]
    y = [np.zeros(B, np.int16) for _ in range(2)]
    assert conv.ProcessMixPcm16(x, 1, 1.0, [0, 1, 0, 1], 0, y, 1, 1.0, B)[0] == cv.AMF_INVALID_ARG
    assert conv.ProcessMixPcm16(x, 1, 1.0, [0, 1, 0, 2], 2, y, 1, 1.0, B)[0] == cv.AMF_INVALID_ARG
    assert conv.ProcessMixPcm16(x, 1, 1.0, [0, 0, 0, 0], 2, y, 1, 1.0, B)[0] == cv.AMF_INVALID_ARG  # empty group
    assert conv.ProcessMixPcm16(x, 1, 0.0, [0, 1, 0, 1], 2, y, 1, 1.0, B)[0] == cv.AMF_INVALID_ARG
    rc, clip, done = conv.ProcessMixPcm16(x, 1, 1.0, [0, 1, 0, 1], 2, y, 1, 1.0, B)
    assert rc == 0 and done == B and not clip
    td = cv.TANConvolution(tan_ctx)
    assert td.Init(cv.TAN_CONVOLUTION_METHOD_TIME_DOMAIN, L, B, C) == 0
    assert td.ProcessMixPcm16(x, 1, 1.0, [0, 1, 0, 1], 2, y, 1, 1.0, B)[0] == cv.AMF_NOT_SUPPORTED
    conv.Release()
    td.Release()
