"""CPU tests of the oracle itself: the C++ restatement of TAN's CPU path and the
FP64 statement, pinned against the reference's delta-IR fixtures
(tan/tests/src/TALibTestConvolution/testresponse.wav) and against each other."""
import numpy as np
import pytest

from oracle import fp64, ref
from tests import helpers as H


def test_fp64_fft_matches_direct_sum():
    g = H.rng(1)
    x = H.noise(g, 1, 5000)[0]
    h = H.irs(g, 1, 3000)[0]
    idx = g.integers(0, 5000, 1000)
    assert np.max(np.abs(fp64.direct_fp64(x, h, idx) - fp64.conv_fp64(x, h)[idx])) < 1e-12


@pytest.mark.parametrize("N", [64, 128, 1024, 4096])
def test_restated_fft_matches_numpy(N):
    g = H.rng(N)
    x = g.standard_normal(N).astype(np.float32)
    re, im = ref.rfft(x)
    X = np.fft.rfft(x.astype(np.float64))
    scale = np.sqrt(N)
    assert np.max(np.abs(re - X.real)) / scale < 1e-5
    assert np.max(np.abs(im - X.imag)) / scale < 1e-5
    y = ref.irfft(re, im)
    assert np.max(np.abs(y - x)) < 1e-5


def test_known_answer_delta_irs_from_reference_fixture():
    """testresponse.wav: ch0 = 0.9 at n=10; ch1 = 0.9@10 + 0.5@1210 + 0.25@2410.
    The output must be the input delayed and scaled, to FP32 rounding."""
    h = H.delta_irs()
    taps = H.golden_taps()["channels"]
    assert [t["index"] for t in taps[1]] == [10, 1210, 2410]
    x = H.pulsetrain(2)
    B = 128  # the reference's test block size (TALibTestConvolution.cpp:92)
    L = h.shape[1]
    conv = ref.RefConvolution(L, B, 2, threads=2)
    y, codes = H.run_stream(conv, x, B, events={0: (h, None)})
    assert all(c == 0 for c in codes)
    T = y.shape[1]
    for c in range(2):
        exp = np.zeros(T, np.float64)
        for t in taps[c]:
            exp[t["index"]:] += t["value"] * x[c, : T - t["index"]].astype(np.float64)
        # block 0 is the crossfade from the initial zero IR
        w = np.arange(B) / B
        exp[:B] *= w
        assert np.max(np.abs(y[c] - exp)) < 2e-6


@pytest.mark.parametrize("C,B,L,swaps", [(2, 256, 2000, [0, 7]), (3, 128, 1024, [0, 3, 4, 9]),
                                         (1, 512, 512, [0, 5]), (2, 64, 5000, [2, 11]),
                                         (2, 256, 400, [0, 6])])  # two partitions
def test_restatement_matches_fp64_with_swaps(C, B, L, swaps):
    g = H.rng(C * 1000 + B)
    nb = 14
    x = H.noise(g, C, nb * B)
    events, fp_events = {}, []
    for k in swaps:
        h = H.irs(g, C, L, (0.1, 0.5))
        events[k] = (h, None)
        fp_events.append((k, {c: h[c] for c in range(C)}))
    conv = ref.RefConvolution(L, B, C, threads=2)
    y, codes = H.run_stream(conv, x, B, events)
    exp = fp64.stream_fp64(x, B, fp_events)
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120


def test_restatement_partial_update_and_flush():
    """UpdateResponseTD with STOP_INPUT on one channel keeps its IR;
    FLUSH_STREAM clears history (intended semantics)."""
    g = H.rng(7)
    C, B, L, nb = 2, 128, 700, 16
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    conv = ref.RefConvolution(L, B, C)
    events = {0: (h0, None), 5: (h1, np.array([0, 1], np.uint32)), 9: (h1, np.array([1, 0], np.uint32))}
    y, _ = H.run_stream(conv, x, B, events)
    # channel 0 took h1 at block 5; channel 1 kept h0 then took h1 at block 9
    exp = fp64.stream_fp64(x, B, [(0, {0: h0[0], 1: h0[1]}), (5, {0: h1[0]}), (9, {1: h1[1]})])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120

    conv = ref.RefConvolution(L, B, C)
    flags = [None] * nb
    for k in range(nb):
        flags[k] = np.array([2 if k == 6 else 0, 0], np.uint32)
    y, _ = H.run_stream(conv, x, B, {0: (h0, None)}, flags_per_block=flags)
    exp = fp64.stream_fp64(x, B, [(0, {0: h0[0], 1: h0[1]})], flush_events=[(6, [0])])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120


def test_restatement_stop_input_ring_out_and_free_channel():
    """STOP_INPUT keeps a channel running for nextpow2(L) samples, then flushes
    it and reports it free (ConvolutionImpl.cpp:2867-2907, 1084-1110)."""
    g = H.rng(11)
    C, B, L = 2, 128, 512  # nextpow2(L) = 512 -> 4 ring-out blocks
    conv = ref.RefConvolution(L, B, C)
    assert conv.update_response_td(H.irs(g, C, L)) == 0
    stop = np.array([1, 0], np.uint32)
    x = H.noise(g, C, B)
    rc, _, done = conv.process(x, None)
    assert rc == 0 and done == B
    assert conv.next_free_channel(stop) == (11, 0xFFFFFFFF)
    for k in range(4):
        rc, y, done = conv.process(x, stop)
        assert rc == 0
    assert conv.next_free_channel(stop) == (0, 0)
    # a free channel's output row is left untouched
    sentinel = np.full((C, B), 7.0, np.float32)
    rc, y, _ = conv.process(x, stop, sentinel.copy())
    assert rc == 0 and np.all(y[0] == 7.0) and not np.all(y[1] == 7.0)
    # all channels stopped and rung out -> AMF_WRONG_STATE
    conv2 = ref.RefConvolution(L, B, 1)
    rc, _, _ = conv2.process(H.noise(g, 1, B), np.array([3], np.uint32))
    assert rc == 15


def test_restatement_free_channel_restarts_from_silence():
    """Stop -> ring-out (input still applied) -> flushed on the last ring-out
    block -> free (output untouched) -> running again from silence."""
    g = H.rng(12)
    C, B, L, nb = 2, 128, 500, 24  # nextpow2(L) = 512: ring-out of 4 blocks
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    flags = [np.array([1 if 5 <= k < 15 else 0, 0], np.uint32) for k in range(nb)]
    conv = ref.RefConvolution(L, B, C)
    assert conv.update_response_td(h) == 0
    y = np.full((C, nb * B), 9.0, np.float32)
    for k in range(nb):
        ys = y[:, k * B:(k + 1) * B].copy()
        rc, ys, _ = conv.process(np.ascontiguousarray(x[:, k * B:(k + 1) * B]), flags[k], ys)
        assert rc == 0
        y[:, k * B:(k + 1) * B] = ys
    # ring-out blocks 5..8, flush before block 8, free 9..14, restart (flush) at 15
    exp = fp64.stream_fp64(x, B, [(0, {0: h[0], 1: h[1]})], flush_events=[(8, [0]), (15, [0])])
    live = np.ones(nb * B, bool)
    live[9 * B:15 * B] = False
    assert np.all(y[0, ~live] == 9.0)
    assert fp64.error_db(y[0, live], exp[0, live]) < -120
    assert fp64.error_db(y[1], exp[1]) < -120


def test_restatement_at_the_bench_shape_matches_fp64():
    """64 channels, B = 512, IR 65536 (128 partitions), a swap at block 33."""
    C, B, L, nb = 64, 512, 65536, 40
    g = H.rng(20261203 + 1)
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L, (0.2, 1.5)), H.irs(g, C, L, (0.2, 1.5))
    conv = ref.RefConvolution(L, B, C, threads=4)
    y, codes = H.run_stream(conv, x, B, {0: (h0, None), 33: (h1, None)}, per_call_blocks=1)
    conv.close()
    assert all(c == 0 for c in codes)
    exp = fp64.stream_fp64(x, B, [(0, {c: h0[c] for c in range(C)}), (33, {c: h1[c] for c in range(C)})])
    assert max(fp64.error_db(y[c], exp[c]) for c in range(C)) < -120


def test_restatement_on_the_dense_ir_fixture_matches_fp64():
    """The reference's dense IR fixture (testresponse2.wav, first 4096 taps) on
    its pulse-train input at the reference test's block size 128."""
    import os

    h = np.load(os.path.join(H.GOLDEN, "testresponse2_head.npy")).astype(np.float32) / 32768.0
    x = H.pulsetrain(2)
    B, L = 128, h.shape[1]
    conv = ref.RefConvolution(L, B, 2, threads=2)
    y, codes = H.run_stream(conv, x, B, {0: (h, None)})
    conv.close()
    assert all(c == 0 for c in codes)
    exp = fp64.stream_fp64(x, B, [(0, {0: h[0], 1: h[1]})])
    for c in range(2):
        assert fp64.error_db(y[c], exp[c]) < -120
