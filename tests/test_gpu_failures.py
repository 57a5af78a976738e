"""Failure detection and injected faults, in forms that fault, trap or hang no
GPU. The reference waits without bound for a pending IR
(tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:425-428) and
up to 50 ms with BLOCK_UNTIL_READY (:686-692); here every device wait is
bounded:

* the tail's bulk-copy pipeline gives up a stage wait after a bound the test
  lowers to zero polls: the kernel records the error, drains its copies in
  flight with the full bound and exits; the host reports AMF_FAIL; a fresh
  object then processes correctly;
* host-side injections on the batched engine: a session closed right after its
  crossfade block, an IR update superseded before it took effect, admission
  refused under churn; the other sessions' outputs are unaffected.
"""
import numpy as np
import pytest

from oracle import ref
from tan_b200 import convolution as cv
from tan_b200 import engine as eng
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def bulk_tiling_index(ctx, B):
    """Index of a compiled cp.async.bulk tail tiling usable at block B."""
    idx = 0
    while True:
        conv = cv.TANConvolution(ctx)
        assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, 4 * B, B, 1) == 0
        rc, t = conv.tiling(idx)
        conv.Release()
        if rc != cv.AMF_OK:
            return None
        # kind-1 tilings are the last entries; their first field is half the slice width
        if idx >= 12 and 2 * t[0] <= B:
            return idx
        idx += 1


def test_bulk_wait_timeout_is_reported_and_a_fresh_object_works(tan_ctx):
    g = H.rng(20261203 + 41)
    C, B, L, nb = 2, 256, 20000, 6
    idx = bulk_tiling_index(tan_ctx, B)
    assert idx is not None
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    conv = cv.TANConvolution(tan_ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    assert conv.tiling(idx)[0] == cv.AMF_OK
    assert cv.lib().tanb_convolution_set_wait_limit(conv._h, 0) == cv.AMF_OK
    assert conv.UpdateResponseTD(h, L) == 0
    codes = []
    for k in range(nb):
        xs = np.ascontiguousarray(x[:, k * B:(k + 1) * B])
        rc, _ = conv.Process(xs, np.zeros_like(xs), B)
        codes.append(rc)
    codes.append(conv.Synchronize())
    assert cv.AMF_FAIL in codes, codes
    assert "timed out" in cv.last_error()
    conv.Release()
    # the context is intact: a fresh object with the same tiling is correct
    fresh = cv.TANConvolution(tan_ctx)
    assert fresh.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    assert fresh.tiling(idx)[0] == cv.AMF_OK
    y, codes = H.run_stream(fresh, x, B, {0: (h, None)})
    assert all(c == 0 for c in codes) and fresh.Synchronize() == 0
    fresh.Release()
    oracle = ref.RefConvolution(L, B, C, threads=2)
    yr, _ = H.run_stream(oracle, x, B, {0: (h, None)})
    oracle.close()
    assert H.rel_err(y, yr) < TOL


def alone(ctx, x, B, events):
    C = x.shape[0]
    L = max(ir.shape[1] for ir in events.values())
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    y, codes = H.run_stream(conv, x, B, {k: (ir, None) for k, ir in events.items()})
    conv.Release()
    return y


def test_engine_session_closed_after_its_crossfade_block(tan_ctx):
    """Session A swaps IRs at block 10 and closes right after that block; B
    runs on; C opens in A's freed slots at block 12. B and C equal themselves
    alone, and A's output up to its close equals A alone."""
    g = H.rng(20261203 + 42)
    B, nb = 256, 30
    xa, xb, xc = H.noise(g, 2, nb * B), H.noise(g, 1, nb * B), H.noise(g, 2, nb * B)
    ha = {0: H.irs(g, 2, 9000), 10: H.irs(g, 2, 9000)}
    hb = {0: H.irs(g, 1, 20000), 10: H.irs(g, 1, 20000)}
    hc = {0: H.irs(g, 2, 9000)}
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=64 << 20, max_channels=4)
    rc, sa = e.open_session(2, 9000)
    rc2, sb = e.open_session(1, 20000)
    assert rc == 0 and rc2 == 0
    ya, yb, yc = np.zeros_like(xa), np.zeros_like(xb), np.zeros((2, (nb - 12) * B), np.float32)
    sc = None
    for k in range(nb):
        if k in ha and sa:
            assert sa.update_response_td(ha[k], block_until_ready=True) == 0
        if k in hb:
            assert sb.update_response_td(hb[k], block_until_ready=True) == 0
        if k == 12:
            rc, sc = e.open_session(2, 9000)
            assert rc == 0 and sc.first_slot == 0  # A's slots
            assert sc.update_response_td(hc[0], block_until_ready=True) == 0
        if sa:
            e.inp[sa.slots] = xa[:, k * B:(k + 1) * B]
        if sc:
            e.inp[sc.slots] = xc[:, (k - 12) * B:(k - 11) * B]
        e.inp[sb.slots] = xb[:, k * B:(k + 1) * B]
        assert e.process() == 0
        if sa:
            ya[:, k * B:(k + 1) * B] = e.out[sa.slots]
        if sc:
            yc[:, (k - 12) * B:(k - 11) * B] = e.out[sc.slots]
        yb[:, k * B:(k + 1) * B] = e.out[sb.slots]
        if k == 10:
            assert sa.close() == 0
            sa = None
    e.release()
    ref_a = alone(tan_ctx, xa[:, :11 * B], B, ha)
    assert H.rel_err(ya[:, :11 * B], ref_a) <= TOL
    assert H.rel_err(yb, alone(tan_ctx, xb, B, hb)) <= TOL
    assert H.rel_err(yc, alone(tan_ctx, xc[:, :(nb - 12) * B], B, hc)) <= TOL


def test_engine_update_superseded_before_it_took_effect(tan_ctx):
    """Two updates between blocks: the first is never heard, the second takes
    effect (with the crossfade) at the next block."""
    g = H.rng(20261203 + 43)
    B, nb, C, L = 256, 20, 2, 12000
    x = H.noise(g, C, nb * B)
    h0, h1, h2 = H.irs(g, C, L), H.irs(g, C, L), H.irs(g, C, L)
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=64 << 20, max_channels=4)
    rc, s = e.open_session(C, L)
    assert rc == 0
    y = np.zeros_like(x)
    for k in range(nb):
        if k == 0:
            assert s.update_response_td(h0, block_until_ready=True) == 0
        if k == 8:
            assert s.update_response_td(h1, block_until_ready=True) == 0
            assert s.update_response_td(h2, block_until_ready=True) == 0
        e.inp[s.slots] = x[:, k * B:(k + 1) * B]
        assert e.process() == 0
        y[:, k * B:(k + 1) * B] = e.out[s.slots]
    assert s.state()["last_swap_block"] == 8
    e.release()
    assert H.rel_err(y, alone(tan_ctx, x, B, {0: h0, 8: h2})) <= TOL


def test_engine_admission_refused_under_churn(tan_ctx):
    """One block per step: a session of 1-3 channels tries to open; when the
    budget refuses it (AMF_OUT_OF_MEMORY) the oldest session leaves. Every
    session's recorded output, from its first block to the last (or its
    close), equals that session alone."""
    g = H.rng(20261203 + 44)
    B, L, steps = 256, 30000, 40
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=24 << 20, max_channels=64)
    live, done, refused = [], [], 0
    for k in range(steps):
        C = int(g.integers(1, 4))
        rc, s = e.open_session(C, L)
        if rc != cv.AMF_OK:
            assert rc == cv.AMF_OUT_OF_MEMORY
            refused += 1
            if live:  # churn: the oldest leaves
                old = live.pop(0)
                assert old["s"].close() == 0
                done.append(old)
        else:
            h = H.irs(g, C, L)
            assert s.update_response_td(h, block_until_ready=True) == 0
            live.append({"s": s, "events": {0: h}, "x": [], "y": []})
        for d in live:
            xb = H.noise(g, d["s"].channels, B)
            d["x"].append(xb)
            e.inp[d["s"].slots] = xb
        assert e.process() == 0
        for d in live:
            d["y"].append(e.out[d["s"].slots].copy())
    e.release()
    assert refused > 0 and live and done
    for d in live + done:
        x, y = np.concatenate(d["x"], axis=1), np.concatenate(d["y"], axis=1)
        assert H.rel_err(y, alone(tan_ctx, x, B, d["events"])) <= TOL
