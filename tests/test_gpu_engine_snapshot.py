"""Engine session snapshot and restore (a session moved between engines, on
one GPU here; between GPUs the restore is the same host-to-device copy): the
restored session continues with the output of the session that never moved,
bit for bit -- with IR swaps before and after the move, an update staged but
not yet in effect at the move, other sessions in both engines, and the two
engines' block counters of either parity (the partial-sum rows alternate with
it)."""
import numpy as np
import pytest

from tan_b200 import convolution as cv
from tan_b200 import engine as eng
from tests import helpers as H

pytestmark = pytest.mark.gpu


def run(engine, sess, x, B, k0, k1, events, others=()):
    """Blocks [k0, k1) of session `sess` (input x, IR events {block: ir} with
    BLOCK_UNTIL_READY); `others` are (session, input) pairs run beside it."""
    y = np.zeros((sess.channels, (k1 - k0) * B), np.float32)
    for k in range(k0, k1):
        if k in events:
            assert sess.update_response_td(events[k], block_until_ready=True) == cv.AMF_OK
        engine.inp[sess.slots] = x[:, k * B:(k + 1) * B]
        for o, xo in others:
            engine.inp[o.slots] = xo[:, (k % 8) * B:(k % 8 + 1) * B]
        assert engine.process() == cv.AMF_OK, cv.last_error()
        y[:, (k - k0) * B:(k - k0 + 1) * B] = engine.out[sess.slots]
    return y


@pytest.mark.parametrize("spectrum,target_pre", [(eng.SPECTRUM_FP32, 2), (eng.SPECTRUM_FP32, 3),
                                                 (eng.SPECTRUM_FP16, 2), (eng.SPECTRUM_FP24, 2)])
def test_restored_session_continues_bit_for_bit(tan_ctx, spectrum, target_pre):
    g = H.rng(20261204 + 40 + target_pre + 10 * spectrum)
    B, C, L, nb, cut = 256, 3, 30000, 50, 25
    x = H.noise(g, C, nb * B)
    h0, h1, hs, h2 = (H.irs(g, C, L) for _ in range(4))
    xo = H.noise(g, 2, 8 * B)
    mk = lambda: eng.Engine(tan_ctx, B, spectrum, budget_bytes=1 << 30, max_channels=16, partitions_per_item=16)

    ref_e = mk()
    rc, s_ref = ref_e.open_session(C, L)
    assert rc == cv.AMF_OK
    y_ref = run(ref_e, s_ref, x, B, 0, nb, {0: h0, 12: h1, cut: hs, 36: h2})
    ref_e.release()

    a = mk()
    rc, other_a = a.open_session(2, 9000)
    assert rc == cv.AMF_OK and other_a.update_response_td(H.irs(g, 2, 9000), block_until_ready=True) == 0
    rc, s_a = a.open_session(C, L)
    assert rc == cv.AMF_OK
    y_a = run(a, s_a, x, B, 0, cut, {0: h0, 12: h1}, [(other_a, xo)])
    # staged, not yet in effect: lands on the first block after the move
    assert s_a.update_response_td(hs, block_until_ready=True) == cv.AMF_OK
    assert s_a.state()["staged"]
    rc, snap = s_a.snapshot()
    assert rc == cv.AMF_OK, cv.last_error()
    assert s_a.close() == cv.AMF_OK
    a.release()

    b = mk()
    rc, other_b = b.open_session(1, 5000)
    assert rc == cv.AMF_OK and other_b.update_response_td(H.irs(g, 1, 5000), block_until_ready=True) == 0
    run(b, other_b, H.noise(g, 1, target_pre * B), B, 0, target_pre, {})  # the target's own block count
    rc, s_b = b.open_session_restore(snap)
    assert rc == cv.AMF_OK, cv.last_error()
    assert (s_b.channels, s_b.ir_length) == (C, L)
    y_b = run(b, s_b, x, B, cut, nb, {36: h2}, [(other_b, H.noise(g, 1, 8 * B))])
    b.release()
    assert np.array_equal(y_a, y_ref[:, :cut * B])
    assert np.array_equal(y_b, y_ref[:, cut * B:])


def test_session_snapshot_rules(tan_ctx):
    g = H.rng(20261204 + 50)
    e = eng.Engine(tan_ctx, 256, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=16)
    rc, s = e.open_session(2, 9000)
    assert rc == cv.AMF_OK and s.update_response_td(H.irs(g, 2, 9000), block_until_ready=True) == 0
    rc, snap = s.snapshot()
    assert rc == cv.AMF_OK
    other = eng.Engine(tan_ctx, 512, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=16)
    assert other.open_session_restore(snap)[0] == cv.AMF_INVALID_ARG  # another block size
    assert e.open_session_restore(snap[:100])[0] == cv.AMF_INVALID_ARG  # short
    bad = snap.copy()
    bad[:8] = 0
    assert e.open_session_restore(bad)[0] == cv.AMF_INVALID_ARG  # not a snapshot
    rc, nu = e.open_session_nu(2, 20000, [(256, 2), (512, 2), (1024, 19)])
    assert rc == cv.AMF_OK, cv.last_error()
    assert nu.snapshot()[0] == cv.AMF_NOT_SUPPORTED
    other.release()
    e.release()
