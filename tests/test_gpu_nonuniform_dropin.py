"""The drop-in TANConvolution with the non-uniform methods
(TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_NONUNIFORM and the GPU names
FHT/FFT_NONUNIFORM_PARTITIONED): levels of growing block size along the IR on
a private engine session. Against the oracle's restatement of the reference's
CPU path (the same convolution, channel flags and crossfade; <= 1e-5 x rms on
every block) and the FP64 statement (<= -120 dB), through the C ABI with host
rows, device rows and multi-block calls."""
import numpy as np
import pytest

from oracle import fp64, ref
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5
NU_METHODS = [cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_NONUNIFORM, cv.TAN_CONVOLUTION_METHOD_FHT_NONUNIFORM_PARTITIONED,
              cv.TAN_CONVOLUTION_METHOD_FFT_NONUNIFORM_PARTITIONED]


def make(ctx, L, B, C, method=cv.TAN_CONVOLUTION_METHOD_FFT_NONUNIFORM_PARTITIONED, levels=None):
    conv = cv.TANConvolution(ctx)
    rc = conv.InitNonUniform(method, L, B, C, levels) if levels else conv.Init(method, L, B, C)
    assert rc == cv.AMF_OK, (rc, cv.last_error())
    return conv


@pytest.mark.parametrize("method", NU_METHODS)
def test_nonuniform_methods_match_restatement_with_swaps(tan_ctx, method):
    g = H.rng(20261203 + 31 + method)
    C, B, L, nb = 3, 256, 20000, 90
    x = H.noise(g, C, nb * B)
    events = {0: (H.irs(g, C, L, (0.2, 1.5)), None), 9: (H.irs(g, C, L, (0.2, 1.5)), None),
              47: (H.irs(g, C, L, (0.2, 1.5)), None)}
    conv = make(tan_ctx, L, B, C, method)
    y, codes = H.run_stream(conv, x, B, events, per_call_blocks=3)
    conv.Release()
    assert all(c == 0 for c in codes)
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, events)
    oracle.close()
    assert H.rel_err(y, yr) < TOL
    exp = fp64.stream_fp64(x, B, [(k, {c: ir[c] for c in range(C)}) for k, (ir, _) in events.items()])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120


def test_nonuniform_flags_and_partial_updates_match_restatement(tan_ctx):
    """STOP_INPUT ring-out and release, FLUSH_STREAM, a partial IR update that
    skips a stopping channel, free channels left untouched and restarting from
    silence (no IR update while a channel is free)."""
    g = H.rng(20261203 + 32)
    C, B, L, nb = 4, 128, 5000, 100  # nextpow2(L) = 8192: a ring-out of 64 blocks
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    events = {0: (h0, None), 7: (h1, np.array([0, 1, 0, 0], np.uint32))}
    flags = []
    for k in range(nb):
        f = np.zeros(C, np.uint32)
        if 3 <= k < 80:
            f[1] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT  # rings out blocks 3..66, free 67..79, restarts 80
        if k == 30:
            f[2] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_FLUSH_STREAM
        if 50 <= k < 60:
            f[3] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT | cv.TAN_CONVOLUTION_CHANNEL_FLAG_FLUSH_STREAM
        flags.append(f)
    sentinel = 3.25
    outs = []
    for kind in ("gpu", "oracle"):
        conv = make(tan_ctx, L, B, C) if kind == "gpu" else ref.RefConvolution(L, B, C)
        y = np.full((C, nb * B), sentinel, np.float32)
        for k in range(nb):
            if k == 70:  # channel 1 rang out and is free
                free = conv.GetNextFreeChannel(flags[k]) if kind == "gpu" else conv.next_free_channel(flags[k])
                assert free == (0, 1), (kind, free)
            if k in events:
                ir, fl = events[k]
                rc = conv.UpdateResponseTD(ir, L, fl) if kind == "gpu" else conv.update_response_td(ir, fl)
                assert rc == 0
            xs = np.ascontiguousarray(x[:, k * B:(k + 1) * B])
            ys = np.ascontiguousarray(y[:, k * B:(k + 1) * B])
            if kind == "gpu":
                rc, done = conv.Process(xs, ys, B, flags[k])
            else:
                rc, ys, done = conv.process(xs, flags[k], ys)
            assert rc == 0 and done == B
            y[:, k * B:(k + 1) * B] = ys
        if kind == "gpu":
            conv.Release()
        else:
            conv.close()
        outs.append(y)
    y, yr = outs
    assert np.array_equal(y == sentinel, yr == sentinel)
    live = yr != sentinel
    assert np.max(np.abs(y[live] - yr[live])) < TOL * np.sqrt(np.mean(yr[live].astype(np.float64) ** 2))


def test_nonuniform_device_rows_equal_host_rows(tan_ctx):
    """Device rows in multi-block calls, host-to-device calls and host rows give
    the same samples bit for bit; an explicit schedule through InitNonUniform."""
    import torch

    g = H.rng(20261203 + 33)
    C, B, L, nb = 2, 128, 30000, 72
    levels = [(128, 2), (256, 2), (512, 2), (1024, 2), (2048, 14)]
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    host = make(tan_ctx, L, B, C, levels=levels)
    y0, codes = H.run_stream(host, x, B, {0: (h0, None), 40: (h1, None)})
    host.Release()
    assert all(c == 0 for c in codes)
    dev = make(tan_ctx, L, B, C, levels=levels)
    hyb = make(tan_ctx, L, B, C, levels=levels)
    xd = torch.from_numpy(x).cuda()
    yd, yh = torch.zeros_like(xd), torch.zeros_like(xd)
    for k0, k1, h in ((0, 40, h0), (40, nb, h1)):
        assert dev.UpdateResponseTDDevice(torch.from_numpy(h).cuda(), L) == 0
        assert hyb.UpdateResponseTD(h, L) == 0
        for a in range(k0, k1, 5):
            b = min(k1, a + 5)
            rc, done = dev.ProcessDevice([xd[c, a * B:b * B] for c in range(C)], [yd[c, a * B:b * B] for c in range(C)],
                                         (b - a) * B)
            assert rc == 0 and done == (b - a) * B
            rc, done = hyb.ProcessHostToDevice(np.ascontiguousarray(x[:, a * B:b * B]),
                                               [yh[c, a * B:b * B] for c in range(C)], (b - a) * B)
            assert rc == 0 and done == (b - a) * B
    assert dev.Synchronize() == 0 and hyb.Synchronize() == 0
    assert np.array_equal(yd.cpu().numpy(), y0)
    assert np.array_equal(yh.cpu().numpy(), y0)
    dev.Release()
    hyb.Release()
    exp = fp64.stream_fp64(x, B, [(0, {c: h0[c] for c in range(C)}), (40, {c: h1[c] for c in range(C)})])
    for c in range(C):
        assert fp64.error_db(y0[c], exp[c]) < -120


def test_nonuniform_init_rules(tan_ctx):
    conv = cv.TANConvolution(tan_ctx)
    # blocks outside the engine's range are refused, not run as uniform
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_NONUNIFORM_PARTITIONED, 20000, 64, 2) == cv.AMF_NOT_SUPPORTED
    assert "non-uniform" in cv.last_error()
    assert conv.InitNonUniform(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, 20000, 256, 2,
                               [(256, 2), (512, 40)]) == cv.AMF_INVALID_ARG
    assert conv.InitNonUniform(cv.TAN_CONVOLUTION_METHOD_FFT_NONUNIFORM_PARTITIONED, 20000, 256, 2,
                               [(256, 2), (512, 4)]) == cv.AMF_INVALID_ARG  # does not cover the IR
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FHT_NONUNIFORM_PARTITIONED, 20000, 256, 2) == cv.AMF_OK
    assert conv.info()["partitions"] == 2  # the base level of the default schedule
    x = np.zeros((2, 256), np.float32)
    rc, _, _ = conv.ProcessMixPcm16([np.zeros(256, np.int16)] * 2, 1, 1.0, np.zeros(2, np.uint32), 1,
                                    [np.zeros(256, np.int16)], 1, 1.0, 256)
    assert rc == cv.AMF_NOT_SUPPORTED
    rc, done = conv.Process(x, x.copy(), 256)
    assert rc == cv.AMF_OK and done == 256, cv.last_error()
    assert conv.ProcessFinalize() == cv.AMF_OK
    conv.Release()
