"""Process and UpdateResponseTD on two threads. In the reference neither
call runs in parallel with itself, but the two may run on different threads
(tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.h:212-216,
separate update and process sections).

Calls on one object take turns, so the output of a threaded run equals a
serial run in which each update lands before some block. The first test
finds that block by comparing against the FP64 statement for every
candidate; the second checks that after a burst of updates the output
settles on the last IR with the whole input history (a swap applies the new
response to the delay line, so later blocks do not depend on when the
earlier updates landed)."""
import threading

import numpy as np
import pytest

from oracle import fp64
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu

C, B, L = 2, 256, 2048


def _conv(ctx):
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == cv.AMF_OK, cv.last_error()
    return conv


def _run(conv, x, h0, worker, after_join):
    """Processes x block by block on this thread while `worker` runs on a
    second one; keeps going for `after_join` blocks after it has finished."""
    nb = x.shape[1] // B
    y = np.zeros_like(x)
    assert conv.UpdateResponseTD(h0, L) == cv.AMF_OK
    codes, progress = [], threading.Event()
    t = threading.Thread(target=worker, args=(progress,))
    t.start()
    k, left = 0, None
    while k < nb and (left is None or left > 0):
        xs = np.ascontiguousarray(x[:, k * B:(k + 1) * B])
        ys = np.zeros((C, B), np.float32)
        rc, done = conv.Process(xs, ys, B)
        codes.append(rc)
        y[:, k * B:(k + 1) * B] = ys
        k += 1
        if k == 8:
            progress.set()
        if left is None and not t.is_alive():
            left = after_join
        elif left is not None:
            left -= 1
    t.join()
    assert left is not None and left == 0, "the worker outlived the input"
    assert all(c == cv.AMF_OK for c in codes), codes
    return y[:, :k * B], k


def test_update_from_another_thread_lands_between_blocks(tan_ctx):
    g = H.rng(4242)
    x = H.noise(g, C, 2000 * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    conv = _conv(tan_ctx)
    rcs = []

    def worker(progress):
        progress.wait(30)
        rcs.append(conv.UpdateResponseTD(h1, L))

    y, nb = _run(conv, x, h0, worker, after_join=4)
    assert rcs == [cv.AMF_OK]
    x = x[:, :nb * B]
    best = None
    for k in range(8, nb):
        exp = fp64.stream_fp64(x, B, [(0, {c: h0[c] for c in range(C)}), (k, {c: h1[c] for c in range(C)})])
        err = max(fp64.error_db(y[c], exp[c]) for c in range(C))
        if best is None or err < best[1]:
            best = (k, err)
    assert best[1] < -120, best
    conv.Release()


def test_burst_of_updates_settles_on_the_last_response(tan_ctx):
    g = H.rng(4343)
    x = H.noise(g, C, 2000 * B)
    h0 = H.irs(g, C, L)
    hs = [H.irs(g, C, L) for _ in range(6)]
    conv = _conv(tan_ctx)
    rcs = []

    def worker(progress):
        progress.wait(30)
        for h in hs:
            rcs.append(conv.UpdateResponseTD(h, L))

    y, nb = _run(conv, x, h0, worker, after_join=6)
    assert rcs == [cv.AMF_OK] * len(hs)
    x = np.asarray(x[:, :nb * B], np.float64)
    # the last update lands at block nb - 6 at the latest (the crossfade
    # block); the blocks after it use the last response on the whole history
    for c in range(C):
        full = fp64.conv_fp64(x[c], np.asarray(hs[-1][c], np.float64))[:nb * B]
        seg = slice((nb - 5) * B, nb * B)
        assert fp64.error_db(y[c, seg], full[seg]) < -120
    conv.Release()
