"""GPU parity at the headline workload's full size, long enough that every
delay-line slot is reused: 64 channels, B = 512, IR 65536 (P = 128), an IR
swap every 32 blocks, 224 blocks (the slot ring of 128 spectra wraps 1.75
times, so partitions up to 127 multiply signal and the tail's slot arithmetic
(cur + i - 1) mod P wraps at every start position), and the configuration's
full 2000 blocks. Also an engine session
with P = 256 over 300 blocks, finalize mode against the oracle, and the
reference's dense IR fixture.

Tolerances: max |gpu - restatement| <= 1e-5 x rms(restatement output), block by
block; error vs FP64 <= -120 dB per channel (FP32 spectra).
"""
import os

import numpy as np
import pytest

from oracle import fp64, ref
from tan_b200 import convolution as cv
from tan_b200 import engine as eng
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _blockwise_rel_err(y, yr, B):
    """Largest per-block max |y - yr|, over rms of the whole reference."""
    rms = np.sqrt(np.mean(yr.astype(np.float64) ** 2))
    d = np.abs(y.astype(np.float64) - yr)
    nb = y.shape[1] // B
    return max(float(d[:, k * B:(k + 1) * B].max()) for k in range(nb)) / rms


def _headline_stream(nb, C=64, B=512, L=65536, every=32):
    g = H.rng(20261203 + 1)
    x = H.noise(g, C, nb * B)
    events, fp_events = {}, []
    for k in range(0, nb, every):
        h = H.irs(g, C, L, (0.2, 1.5))
        events[k] = (h, None)
        fp_events.append((k, {c: h[c] for c in range(C)}))
    return x, events, fp_events


def test_headline_shape_ring_wraps_matches_restatement_and_fp64(tan_ctx):
    import torch

    C, B, L, nb = 64, 512, 65536, 224
    x, events, fp_events = _headline_stream(nb, C, B, L)
    oracle = ref.RefConvolution(L, B, C, threads=os.cpu_count() or 4)
    assert oracle.partitions >= 128
    yr, codes = H.run_stream(oracle, x, B, events)
    oracle.close()
    assert all(c == 0 for c in codes)

    # host rows, one block per call, as the plugin API is called
    conv = cv.TANConvolution(tan_ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C) == cv.AMF_OK
    assert conv.info()["partitions"] == 128
    y, codes = H.run_stream(conv, x, B, events)
    assert all(c == 0 for c in codes)
    conv.Release()
    err = _blockwise_rel_err(y, yr, B)
    assert err < TOL, err

    # device rows and device IR rows: the bench's device-resident path
    dev = cv.TANConvolution(tan_ctx)
    assert dev.Init(cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C) == cv.AMF_OK
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    for k in range(nb):
        if k in events:
            assert dev.UpdateResponseTDDevice(torch.from_numpy(events[k][0]).cuda(), L) == 0
        rc, done = dev.ProcessDevice([xd[c, k * B:(k + 1) * B] for c in range(C)],
                                     [yd[c, k * B:(k + 1) * B] for c in range(C)], B)
        assert rc == 0 and done == B
    assert dev.Synchronize() == 0
    dev.Release()
    assert np.array_equal(yd.cpu().numpy(), y)

    exp = fp64.stream_fp64(x, B, fp_events)
    worst = max(fp64.error_db(y[c], exp[c]) for c in range(C))
    assert worst < -120, worst


def test_headline_config_2000_blocks_matches_restatement(tan_ctx):
    """The headline configuration at its stated length: 64 channels, B = 512,
    IR 65536, every channel's IR replaced every 32 blocks (eight IR sets
    cycled), 2000 blocks through the plugin call with page-locked host rows
    (read and written in place by the head), block by block against the
    restatement on every channel; FP64 on two channels over the first 320
    blocks (the FP64 statement convolves the whole stream once per IR
    version)."""
    import torch

    C, B, L, nb, every = 64, 512, 65536, 2000, 32
    g = H.rng(20261203 + 21)
    sets = [H.irs(g, C, L, (0.2, 1.5)) for _ in range(8)]
    tx = torch.from_numpy(H.noise(g, C, nb * B)).pin_memory()
    x = tx.numpy()
    events = {k: (sets[(k // every) % 8], None) for k in range(0, nb, every)}
    oracle = ref.RefConvolution(L, B, C, threads=os.cpu_count() or 4)
    yr, codes = H.run_stream(oracle, x, B, events)
    oracle.close()
    assert all(c == 0 for c in codes)
    ty = torch.zeros((C, nb * B), dtype=torch.float32).pin_memory()
    y = ty.numpy()
    conv = cv.TANConvolution(tan_ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C) == cv.AMF_OK
    in_place = set()
    for k in range(nb):
        if k in events:
            assert conv.UpdateResponseTD(events[k][0], L) == cv.AMF_OK
        rc, done = conv.Process([x[c, k * B:(k + 1) * B] for c in range(C)],
                                [y[c, k * B:(k + 1) * B] for c in range(C)], B)
        assert rc == cv.AMF_OK and done == B
        in_place.add(conv.call_times()["in_place"])
    conv.Release()
    assert in_place == {3}
    err = _blockwise_rel_err(y, yr, B)
    assert err < TOL, err
    n1 = 320
    exp = fp64.stream_fp64(x[:2, :n1 * B], B, [(k, {c: ir[c] for c in range(2)}) for k, (ir, _) in events.items()
                                             if k < n1])
    for c in range(2):
        assert fp64.error_db(y[c, :n1 * B], exp[c]) < -120


def test_engine_session_p256_long_run_mix_equals_alone(tan_ctx):
    """An engine session of 4 channels with P = 256 (IR 65536 at B = 256) over
    300 blocks with swaps, beside two other sessions: equal to the session alone
    through TANConvolution and to FP64."""
    g = H.rng(20261203 + 11)
    B, nb = 256, 300
    specs = [(4, 65536, [0, 70, 200]), (2, 9000, [0, 150]), (1, 40000, [0])]
    sessions = []
    for C, L, swaps in specs:
        sessions.append({"C": C, "L": L, "x": H.noise(g, C, nb * B),
                         "events": {k: H.irs(g, C, L, (0.2, 1.5)) for k in swaps}})
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=16)
    live = []
    for s in sessions:
        rc, sess = engine.open_session(s["C"], s["L"])
        assert rc == 0, cv.last_error()
        live.append(sess)
    outs = [np.zeros((s["C"], nb * B), np.float32) for s in sessions]
    for k in range(nb):
        for s, sess in zip(sessions, live):
            if k in s["events"]:
                assert sess.update_response_td(s["events"][k], block_until_ready=True) == 0
            engine.inp[sess.slots] = s["x"][:, k * B:(k + 1) * B]
        assert engine.process() == 0, cv.last_error()
        for y, sess in zip(outs, live):
            y[:, k * B:(k + 1) * B] = engine.out[sess.slots]
    engine.release()
    s, y = sessions[0], outs[0]
    conv = cv.TANConvolution(tan_ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, s["L"], B, s["C"]) == 0
    assert conv.info()["partitions"] == 256
    ya, codes = H.run_stream(conv, s["x"], B, {k: (ir, None) for k, ir in s["events"].items()})
    conv.Release()
    assert all(c == 0 for c in codes)
    err = _blockwise_rel_err(y, ya, B)
    assert err <= TOL, err
    for s, y in zip(sessions, outs):
        exp = fp64.stream_fp64(s["x"], B, [(k, {c: ir[c] for c in range(s["C"])}) for k, ir in s["events"].items()])
        for c in range(s["C"]):
            assert fp64.error_db(y[c], exp[c]) < -120


@pytest.mark.parametrize("per_call_blocks", [1, 3])
def test_finalize_mode_matches_restatement(tan_ctx, per_call_blocks):
    """USE_PROCESS_FINALIZE (Process returns after the head; ProcessFinalize
    enqueues the tail) against the restatement, with swaps and channel flags."""
    g = H.rng(20261203 + 12)
    C, B, L, nb = 4, 256, 9000, 40
    x = H.noise(g, C, nb * B)
    h0, h1, h2 = H.irs(g, C, L), H.irs(g, C, L), H.irs(g, C, L)
    events = {0: (h0, None), 13: (h1, None), 27: (h2, np.array([0, 1, 0, 0], np.uint32))}
    flags = []
    for k in range(nb):
        f = np.zeros(C, np.uint32)
        if 5 <= k < 12:
            f[2] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT
        if k == 20:
            f[3] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_FLUSH_STREAM
        flags.append(f)
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, events, flags_per_block=flags)
    oracle.close()
    fin = cv.TANConvolution(tan_ctx)
    method = cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM | cv.TAN_CONVOLUTION_METHOD_USE_PROCESS_FINALIZE
    assert fin.Init(method, L, B, C) == 0
    y = np.zeros_like(yr)
    k = 0
    while k < nb:
        if k in events:
            assert fin.UpdateResponseTD(events[k][0], L, events[k][1]) == 0
        step = 1
        if per_call_blocks > 1 and all(not flags[j].any() for j in range(k, min(nb, k + per_call_blocks))):
            step = min(per_call_blocks, nb - k)
            while step > 1 and any(j in events for j in range(k + 1, k + step)):
                step -= 1
        xs = np.ascontiguousarray(x[:, k * B:(k + step) * B])
        ys = np.zeros_like(xs)
        rc, done = fin.Process(xs, ys, step * B, flags[k] if step == 1 else None)
        assert rc == 0 and done == step * B
        assert fin.ProcessFinalize() == 0
        y[:, k * B:(k + step) * B] = ys
        k += step
    fin.Release()
    err = _blockwise_rel_err(y, yr, B)
    assert err < TOL, err


def test_dense_ir_fixture_against_fp64_and_restatement(tan_ctx):
    """The reference's dense IR fixture (testresponse2.wav, first 4096 taps of
    both channels) on its pulse-train input (pulsetrainS.wav), at the
    reference test's block size 128."""
    h = np.load(os.path.join(H.GOLDEN, "testresponse2_head.npy")).astype(np.float32) / 32768.0
    x = H.pulsetrain(2)
    B, L = 128, h.shape[1]
    conv = cv.TANConvolution(tan_ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, 2) == 0
    y, codes = H.run_stream(conv, x, B, {0: (h, None)}, per_call_blocks=4)
    conv.Release()
    assert all(c == 0 for c in codes)
    oracle = ref.RefConvolution(L, B, 2, threads=2)
    yr, _ = H.run_stream(oracle, x, B, {0: (h, None)})
    oracle.close()
    assert H.rel_err(y, yr) < TOL
    exp = fp64.stream_fp64(x, B, [(0, {0: h[0], 1: h[1]})])
    for c in range(2):
        assert fp64.error_db(y[c], exp[c]) < -120
