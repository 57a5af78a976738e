"""Host rows in page-locked memory: when the caller's input and output rows
(and IR rows) sit at one stride in one pinned allocation, Process reads and
writes them in place over the bus and UpdateResponseTD transfers the IR rows
with one strided copy, instead of staging them through the object's own
buffers. The results are bit for bit those of the staged path (pageable rows),
which the parity tests pin to the oracle; rows that alias, scatter over
allocations or are misaligned take the staged path."""
import numpy as np
import pytest

from oracle import ref
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def pinned(shape):
    import torch

    t = torch.zeros(shape, dtype=torch.float32, pin_memory=True)
    return t, t.numpy()


def drive(conv, x_rows, y_rows, B, nb, events, per_call=3, flags=None, in_place_seen=None):
    """Runs nb blocks; x_rows(k0, k1) / y_rows(k0, k1) give the call's row lists."""
    k = 0
    while k < nb:
        if k in events:
            assert conv.UpdateResponseTD(events[k], events[k].shape[1]) == cv.AMF_OK
        step = min(per_call, nb - k)
        while step > 1 and any(j in events for j in range(k + 1, k + step)):
            step -= 1
        rc, done = conv.Process(x_rows(k, k + step), y_rows(k, k + step), step * B, flags)
        assert rc == cv.AMF_OK and done == step * B, cv.last_error()
        if in_place_seen is not None:
            in_place_seen.add(conv.call_times()["in_place"])
        k += step


def make(ctx, L, B, C):
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C) == cv.AMF_OK
    return conv


def test_pinned_rows_equal_staged_rows_and_the_oracle(tan_ctx):
    g = H.rng(20261204 + 1)
    C, B, L, nb = 8, 256, 20000, 40
    x = H.noise(g, C, nb * B)
    irs = {0: H.irs(g, C, L), 17: H.irs(g, C, L)}
    # staged: pageable rows
    conv = make(tan_ctx, L, B, C)
    y0 = np.zeros_like(x)
    seen0 = set()
    drive(conv, lambda a, b: [np.ascontiguousarray(x[c, a * B:b * B]) for c in range(C)],
          lambda a, b: [y0[c, a * B:b * B] for c in range(C)], B, nb, irs, in_place_seen=seen0)
    conv.Release()
    assert seen0 == {0}
    # in place: pinned input, output and IR rows
    tx, xp = pinned((C, nb * B))
    ty, yp = pinned((C, nb * B))
    xp[:] = x
    pins = {}
    for k, h in irs.items():
        th, hp = pinned(h.shape)
        hp[:] = h
        pins[k] = (th, hp)
    conv = make(tan_ctx, L, B, C)
    seen = set()
    drive(conv, lambda a, b: [xp[c, a * B:b * B] for c in range(C)], lambda a, b: [yp[c, a * B:b * B] for c in range(C)],
          B, nb, {k: hp for k, (th, hp) in pins.items()}, in_place_seen=seen)
    conv.Release()
    assert seen == {3}, seen
    assert np.array_equal(yp, y0)
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, {k: (h, None) for k, h in irs.items()})
    oracle.close()
    assert H.rel_err(yp, yr) < TOL


def test_pinned_rows_in_one_long_call(tan_ctx):
    """One Process call of 20 blocks (more than one chunk of staged blocks)
    on page-locked rows equals the same blocks one call each on pageable rows."""
    g = H.rng(20261204 + 4)
    C, B, L, nb = 6, 128, 9000, 20
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    conv = make(tan_ctx, L, B, C)
    assert conv.UpdateResponseTD(h, L) == cv.AMF_OK
    y0 = np.zeros_like(x)
    drive(conv, lambda a, b: [np.ascontiguousarray(x[c, a * B:b * B]) for c in range(C)],
          lambda a, b: [y0[c, a * B:b * B] for c in range(C)], B, nb, {}, per_call=1)
    conv.Release()
    tx, xp = pinned((C, nb * B))
    ty, yp = pinned((C, nb * B))
    xp[:] = x
    conv = make(tan_ctx, L, B, C)
    assert conv.UpdateResponseTD(h, L) == cv.AMF_OK
    rc, done = conv.Process([xp[c] for c in range(C)], [yp[c] for c in range(C)], nb * B)
    assert rc == cv.AMF_OK and done == nb * B
    assert conv.call_times()["in_place"] == 3
    conv.Release()
    assert np.array_equal(yp, y0)


def test_pinned_rows_with_silent_channels_and_flags(tan_ctx):
    """Null input rows read as silence in place too; a channel stopped with
    STOP_INPUT rings out and its output row is left as the staged path leaves it."""
    g = H.rng(20261204 + 2)
    C, B, L, nb = 6, 128, 6000, 30
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    silent = {1, 4}
    outs = []
    for kind in ("staged", "pinned"):
        conv = make(tan_ctx, L, B, C)
        assert conv.UpdateResponseTD(h, L) == cv.AMF_OK
        if kind == "pinned":
            tx, xs = pinned((C, nb * B))
            ty, ys = pinned((C, nb * B))
            xs[:] = x
        else:
            xs, ys = x.copy(), np.zeros((C, nb * B), np.float32)
        ys[:] = 7.5
        seen = set()
        for k in range(nb):
            f = np.zeros(C, np.uint32)
            if k >= 12:
                f[2] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT
            xin = [None if c in silent else (xs[c, k * B:(k + 1) * B] if kind == "pinned"
                                             else np.ascontiguousarray(xs[c, k * B:(k + 1) * B])) for c in range(C)]
            yout = [ys[c, k * B:(k + 1) * B] for c in range(C)]
            rc, done = conv.Process(xin, yout, B, f)
            assert rc == cv.AMF_OK and done == B
            seen.add(conv.call_times()["in_place"])
        conv.Release()
        assert seen == ({3} if kind == "pinned" else {0}), (kind, seen)
        outs.append(np.array(ys))
    assert np.array_equal(outs[0], outs[1])


def test_pinned_rows_that_alias_or_are_misaligned_take_the_staged_path(tan_ctx):
    g = H.rng(20261204 + 3)
    C, B, L, nb = 4, 256, 9000, 12
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    # reference output, block by block through pageable rows
    conv = make(tan_ctx, L, B, C)
    assert conv.UpdateResponseTD(h, L) == cv.AMF_OK
    y0 = np.zeros_like(x)
    drive(conv, lambda a, b: [np.ascontiguousarray(x[c, a * B:b * B]) for c in range(C)],
          lambda a, b: [y0[c, a * B:b * B] for c in range(C)], B, nb, {}, per_call=1)
    conv.Release()
    # in place: output rows are the input rows
    t, buf = pinned((C, nb * B))
    buf[:] = x
    conv = make(tan_ctx, L, B, C)
    assert conv.UpdateResponseTD(h, L) == cv.AMF_OK
    seen = set()
    drive(conv, lambda a, b: [buf[c, a * B:b * B] for c in range(C)], lambda a, b: [buf[c, a * B:b * B] for c in range(C)],
          B, nb, {}, per_call=1, in_place_seen=seen)
    conv.Release()
    assert seen == {0} and np.array_equal(buf, y0)
    # misaligned rows (4 bytes past a 16-byte boundary)
    tx, xp = pinned((C, nb * B + 4))
    ty, yp = pinned((C, nb * B + 4))
    xp[:, 1:1 + nb * B] = x
    conv = make(tan_ctx, L, B, C)
    assert conv.UpdateResponseTD(h, L) == cv.AMF_OK
    seen = set()
    drive(conv, lambda a, b: [xp[c, 1 + a * B:1 + b * B] for c in range(C)],
          lambda a, b: [yp[c, 1 + a * B:1 + b * B] for c in range(C)], B, nb, {}, per_call=1, in_place_seen=seen)
    conv.Release()
    assert seen == {0} and np.array_equal(yp[:, 1:1 + nb * B], y0)
