"""Snapshot and restore of a drop-in object's stream state (checkpoint, or a
session's migration between GPUs through host memory; one GPU here): an
object restored from a snapshot continues the stream with the output of the
uninterrupted object bit for bit -- with IR swaps before and after the cut, a
pending update at the cut, channel flags, multi-block calls and finalize
mode -- and the uninterrupted stream matches the restatement."""
import numpy as np
import pytest

from oracle import ref
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def make(ctx, L, B, C, method=cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED):
    conv = cv.TANConvolution(ctx)
    assert conv.Init(method, L, B, C) == cv.AMF_OK
    return conv


def drive(conv, x, B, k0, k1, events, flags, per_call=1, finalize=False, leave_due=False):
    """Blocks [k0, k1) of the stream; returns their output. leave_due: in
    finalize mode, the last call's ProcessFinalize is left to the caller."""
    C = x.shape[0]
    y = np.zeros((C, (k1 - k0) * B), np.float32)
    k = k0
    while k < k1:
        if k in events:
            assert conv.UpdateResponseTD(events[k], events[k].shape[1]) == cv.AMF_OK
        step = 1
        if per_call > 1 and flags[k] is None:
            step = min(per_call, k1 - k)
            while step > 1 and any(j in events or flags[j] is not None for j in range(k + 1, k + step)):
                step -= 1
        xs = np.ascontiguousarray(x[:, k * B:(k + step) * B])
        ys = np.zeros_like(xs)
        rc, done = conv.Process(xs, ys, step * B, flags[k])
        assert rc == cv.AMF_OK and done == step * B, cv.last_error()
        if finalize and not (leave_due and k + step == k1):
            assert conv.ProcessFinalize() == cv.AMF_OK
        y[:, (k - k0) * B:(k - k0 + step) * B] = ys
        k += step
    return y


@pytest.mark.parametrize("finalize,per_call,cut_pending", [(False, 1, False), (False, 3, True), (True, 1, True)])
def test_restored_object_continues_the_stream(tan_ctx, finalize, per_call, cut_pending):
    g = H.rng(20261204 + 20 + per_call + (2 if finalize else 0))
    C, B, L, nb, cut = 4, 256, 20000, 60, 30
    x = H.noise(g, C, nb * B)
    events = {0: H.irs(g, C, L), 17: H.irs(g, C, L), 44: H.irs(g, C, L)}
    flags = [None] * nb
    for k in range(8, 14):
        f = np.zeros(C, np.uint32)
        f[2] = cv.TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT
        flags[k] = f
    method = cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED
    if finalize:
        method |= cv.TAN_CONVOLUTION_METHOD_USE_PROCESS_FINALIZE
    full = make(tan_ctx, L, B, C, method)
    y_full = drive(full, x, B, 0, nb, events, flags, per_call, finalize)
    full.Release()

    a = make(tan_ctx, L, B, C, method)
    # in finalize mode the cut falls between a Process and its ProcessFinalize
    y_a = drive(a, x, B, 0, cut, events, flags, per_call, finalize, leave_due=True)
    if cut_pending:  # an update made before the cut lands on the restored object's first block
        assert a.UpdateResponseTD(events[17] * 0.5, L) == cv.AMF_OK
    rc, snap = a.Snapshot()
    assert rc == cv.AMF_OK, cv.last_error()
    b = make(tan_ctx, L, B, C, method)
    # b has a history of its own, which the restore replaces
    drive(b, H.noise(g, C, 5 * B), B, 0, 5, {0: H.irs(g, C, L)}, [None] * 5, 1, finalize)
    assert b.Restore(snap) == cv.AMF_OK, cv.last_error()
    rest = {k - cut: ev for k, ev in events.items() if k >= cut}
    xr = np.ascontiguousarray(x[:, cut * B:])
    y_a2 = drive(a, xr, B, 0, nb - cut, rest, flags[cut:], per_call, finalize)
    y_b = drive(b, xr, B, 0, nb - cut, rest, flags[cut:], per_call, finalize)
    a.Release()
    b.Release()
    assert np.array_equal(y_b, y_a2)
    assert np.array_equal(y_a, y_full[:, :cut * B])
    if not cut_pending:
        assert np.array_equal(y_b, y_full[:, cut * B:])
        oracle = ref.RefConvolution(L, B, C, threads=2)
        yr, _ = H.run_stream(oracle, x, B, {k: (ev, None) for k, ev in events.items()}, flags_per_block=flags)
        oracle.close()
        assert H.rel_err(y_full, yr) < TOL


def test_snapshot_rules(tan_ctx):
    g = H.rng(20261204 + 30)
    a = make(tan_ctx, 9000, 256, 2)
    assert a.UpdateResponseTD(H.irs(g, 2, 9000), 9000) == cv.AMF_OK
    rc, snap = a.Snapshot()
    assert rc == cv.AMF_OK
    other = make(tan_ctx, 9000, 512, 2)
    assert other.Restore(snap) == cv.AMF_INVALID_ARG  # another configuration
    assert a.Restore(snap[:-1]) == cv.AMF_INVALID_ARG  # short
    bad = snap.copy()
    bad[:8] = 0
    assert a.Restore(bad) == cv.AMF_INVALID_ARG  # not a snapshot
    td = cv.TANConvolution(tan_ctx)
    assert td.Init(cv.TAN_CONVOLUTION_METHOD_TIME_DOMAIN, 512, 256, 2) == cv.AMF_OK
    assert td.Snapshot()[0] == cv.AMF_NOT_SUPPORTED
    nu = cv.TANConvolution(tan_ctx)
    assert nu.Init(cv.TAN_CONVOLUTION_METHOD_FFT_NONUNIFORM_PARTITIONED, 20000, 256, 2) == cv.AMF_OK
    assert nu.Snapshot()[0] == cv.AMF_NOT_SUPPORTED
    for o in (a, other, td, nu):
        o.Release()
