"""Batched engine on the GPU: sessions with different channel counts and IR
lengths (uneven partition counts) processed together must give, per session,
the same output as that session alone through the single-object path
(tolerance 1e-5 x rms), also when sessions open and close mid-stream; FP16 /
BF16 spectra and the 24-bit form (spectra and delay line) are measured
against the FP64 statement in dB; admission is by the device-memory budget."""
import numpy as np
import pytest

from oracle import fp64
from tan_b200 import convolution as cv
from tan_b200 import engine as eng
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def alone(ctx, x, B, events):
    """The session run by itself through TANConvolution (the plain path)."""
    C, T = x.shape
    L = max(ir.shape[1] for ir in events.values())
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    y, codes = H.run_stream(conv, x, B, {k: (ir, None) for k, ir in events.items()})
    conv.Release()
    return y


def run_engine(engine, sessions, nb, close_at=None, open_late=None):
    """sessions: list of dict(C, L, x, events, start); returns outputs per session."""
    B = engine.block
    outs = [None] * len(sessions)
    live = {}
    for k in range(nb):
        for i, s in enumerate(sessions):
            if s["start"] == k:
                rc, sess = engine.open_session(s["C"], s["L"])
                assert rc == 0, cv.last_error()
                live[i] = sess
                outs[i] = np.zeros((s["C"], (nb - k) * B), np.float32)
            if close_at and close_at.get(i) == k and i in live:
                assert live.pop(i).close() == 0
        for i, sess in live.items():
            s = sessions[i]
            kk = k - s["start"]
            if kk in s["events"]:
                assert sess.update_response_td(s["events"][kk], block_until_ready=True) == 0
            engine.inp[sess.slots] = s["x"][:, kk * B:(kk + 1) * B]
        assert engine.process() == 0, cv.last_error()
        for i, sess in live.items():
            kk = k - sessions[i]["start"]
            outs[i][:, kk * B:(kk + 1) * B] = engine.out[sess.slots]
    return outs


def make_sessions(g, B, specs, nb):
    sessions = []
    for (C, L, start, swaps) in specs:
        n = nb - start
        x = H.noise(g, C, n * B)
        events = {k: H.irs(g, C, L, (0.2, 1.5)) for k in swaps}
        sessions.append({"C": C, "L": L, "x": x, "events": events, "start": start})
    return sessions


def test_engine_mix_equals_alone(tan_ctx):
    g = H.rng(31)
    B, nb = 256, 40
    specs = [(2, 3000, 0, [0, 17]), (1, 20000, 0, [0, 9, 30]), (3, 65536, 3, [0, 11]), (4, 700, 5, [0]),
             (2, 256, 0, [0, 20])]
    sessions = make_sessions(g, B, specs, nb)
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=64, partitions_per_item=16)
    outs = run_engine(engine, sessions, nb)
    for s, y in zip(sessions, outs):
        ya = alone(tan_ctx, s["x"], B, s["events"])
        rms = np.sqrt(np.mean(ya.astype(np.float64) ** 2))
        assert np.max(np.abs(y - ya)) <= TOL * rms
        exp = fp64.stream_fp64(s["x"], B, [(k, {c: ir[c] for c in range(s["C"])}) for k, ir in s["events"].items()])
        for c in range(s["C"]):
            assert fp64.error_db(y[c], exp[c]) < -120
    engine.release()


def test_engine_fp24_mix_equals_each_session_alone(tan_ctx):
    """24-bit spectra and delay line: each session's samples in the mix are the
    samples of that session alone in its own FP24 engine, bit for bit, and
    within -90 dB of the FP64 statement."""
    g = H.rng(36)
    B, nb = 256, 30
    specs = [(2, 3000, 0, [0, 17]), (1, 20000, 0, [0, 9]), (3, 65536, 3, [0, 11]), (2, 256, 0, [0, 20])]
    sessions = make_sessions(g, B, specs, nb)
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP24, budget_bytes=1 << 30, max_channels=64, partitions_per_item=16)
    outs = run_engine(engine, sessions, nb)
    engine.release()
    for s, y in zip(sessions, outs):
        solo = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP24, budget_bytes=1 << 28, max_channels=8, partitions_per_item=16)
        ya = run_engine(solo, [dict(s, start=0)], nb - s["start"])[0]
        solo.release()
        assert np.array_equal(y, ya)
        exp = fp64.stream_fp64(s["x"], B, [(k, {c: ir[c] for c in range(s["C"])}) for k, ir in s["events"].items()])
        for c in range(s["C"]):
            assert fp64.error_db(y[c], exp[c]) < -90


def test_engine_churn_does_not_disturb_other_sessions(tan_ctx):
    g = H.rng(32)
    B, nb = 256, 36
    specs = [(2, 5000, 0, [0, 13]), (1, 9000, 2, [0]), (2, 30000, 4, [0, 20]), (3, 1000, 10, [0, 4])]
    sessions = make_sessions(g, B, specs, nb)
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=256 << 20, max_channels=16, partitions_per_item=8)
    # session 1 closes at block 12, freeing slots/memory that session 3 (opens at 10) and later reuse
    outs = run_engine(engine, sessions, nb, close_at={1: 12})
    for i, (s, y) in enumerate(zip(sessions, outs)):
        if i == 1:
            continue
        ya = alone(tan_ctx, s["x"], B, s["events"])
        rms = np.sqrt(np.mean(ya.astype(np.float64) ** 2))
        assert np.max(np.abs(y - ya)) <= TOL * rms, i
    engine.release()


@pytest.mark.parametrize("spectrum,limit_db", [(eng.SPECTRUM_FP16, -60.0), (eng.SPECTRUM_BF16, -40.0),
                                               (eng.SPECTRUM_FP24, -90.0)])
def test_engine_reduced_precision_spectra_error_db(tan_ctx, spectrum, limit_db):
    g = H.rng(33 + spectrum)
    B, nb = 256, 24
    specs = [(2, 8192, 0, [0]), (2, 40000, 0, [0, 10])]
    sessions = make_sessions(g, B, specs, nb)
    engine = eng.Engine(tan_ctx, B, spectrum, budget_bytes=1 << 28, max_channels=16)
    outs = run_engine(engine, sessions, nb)
    worst = -np.inf
    for s, y in zip(sessions, outs):
        exp = fp64.stream_fp64(s["x"], B, [(k, {c: ir[c] for c in range(s["C"])}) for k, ir in s["events"].items()])
        for c in range(s["C"]):
            worst = max(worst, fp64.error_db(y[c], exp[c]))
    print(f"spectrum {spectrum}: worst channel error vs FP64 {worst:.1f} dB")
    assert worst < limit_db
    engine.release()


def test_engine_admission_by_budget(tan_ctx):
    B = 256
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=32 << 20, max_channels=64)
    opened = []
    while True:
        rc, s = engine.open_session(2, 65536)
        if rc != 0:
            assert rc == cv.AMF_OUT_OF_MEMORY
            break
        opened.append(s)
    assert 1 <= len(opened) < 20
    assert engine.info()["arena_bytes"] <= 32 << 20
    assert opened[0].close() == 0
    rc, s = engine.open_session(2, 65536)
    assert rc == 0
    assert engine.process() == 0
    engine.release()


def test_engine_async_update_from_another_thread(tan_ctx):
    """IR updates issued from a second thread while blocks run: the swap lands
    on the first block after the upload finished (reported by the engine), and
    the output equals the plain path with the swap at that block. Blocks run
    until the swap has landed and 20 more have followed (the upload's timing
    depends on the host's thread scheduling)."""
    import threading

    g = H.rng(34)
    B, C, L, max_blocks = 256, 2, 30000, 3000
    x = H.noise(g, C, max_blocks * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=256 << 20, max_channels=8)
    rc, sess = engine.open_session(C, L)
    assert rc == 0
    assert sess.update_response_td(h0, block_until_ready=True) == 0
    y = np.zeros((C, max_blocks * B), np.float32)
    started = threading.Event()
    results = []

    def worker():
        started.wait()
        results.append(sess.update_response_td(h1))

    t = threading.Thread(target=worker)
    t.start()
    nb = max_blocks
    for k in range(max_blocks):
        if k == 10:
            started.set()
        engine.inp[sess.slots] = x[:, k * B:(k + 1) * B]
        assert engine.process() == 0, cv.last_error()
        y[:, k * B:(k + 1) * B] = engine.out[sess.slots]
        k_swap = sess.state()["last_swap_block"]
        if k_swap > 0 and k >= k_swap + 20:
            nb = k + 1
            break
    t.join()
    assert results == [0]
    st = sess.state()
    k_swap = st["last_swap_block"]
    assert st["blocks"] == nb and 10 <= k_swap < nb and not st["staged"]
    ya = alone(tan_ctx, x[:, :nb * B], B, {0: h0, k_swap: h1})
    rms = np.sqrt(np.mean(ya.astype(np.float64) ** 2))
    assert np.max(np.abs(y[:, :nb * B] - ya)) <= TOL * rms
    engine.release()


def test_engine_device_io_equals_host_io(tan_ctx):
    """process_device (device rows, stride ld) and process (pinned host
    buffers) run the same block launch: outputs are bit-identical, also on a
    swap block and for sessions with P <= 2 (no work items)."""
    import torch

    g = H.rng(35)
    B, nb = 256, 20
    specs = [(2, 9000), (1, 700), (3, 40000), (1, 256)]
    irs0 = [H.irs(g, C, L) for C, L in specs]
    irs1 = [H.irs(g, C, L) for C, L in specs]
    engines, sess = [], []
    for _ in range(2):
        e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=256 << 20, max_channels=16, partitions_per_item=8)
        ss = []
        for C, L in specs:
            rc, s = e.open_session(C, L)
            assert rc == 0
            ss.append(s)
        engines.append(e)
        sess.append(ss)
    nslots = engines[0].info()["slot_hwm"]
    x = H.noise(g, nslots, nb * B)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    yh = np.zeros_like(x)
    for k in range(nb):
        for j in range(len(specs)):
            for e, ss in zip(engines, sess):
                if k in (0, 9):
                    ir = irs0[j] if k == 0 else irs1[j]
                    assert ss[j].update_response_td(ir, block_until_ready=True) == 0
        engines[0].inp[:nslots] = x[:, k * B:(k + 1) * B]
        assert engines[0].process() == 0
        yh[:, k * B:(k + 1) * B] = engines[0].out[:nslots]
        assert engines[1].process_device(xd.data_ptr() + k * B * 4, yd.data_ptr() + k * B * 4, nb * B) == 0, \
            cv.last_error()
    assert engines[1].synchronize() == 0
    assert np.array_equal(yd.cpu().numpy(), yh)
    for e in engines:
        e.release()


def test_engine_write_input_rows(tan_ctx):
    """write_input copies block samples of strided rows into the input buffer
    at consecutive slots (threaded above 1 MB) and refuses slots out of range."""
    B = 256
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=64 << 20, max_channels=2048)
    g = H.rng(36)
    x = H.noise(g, 1500, 3 * B)  # rows longer than a block: ld = 3B
    assert e.write_input(5, x) == 0
    assert np.array_equal(e.inp[5:1505], x[:, :B])
    small = H.noise(g, 3, B)
    assert e.write_input(0, small) == 0
    assert np.array_equal(e.inp[0:3], small)
    assert e.write_input(2047, small) == cv.AMF_INVALID_ARG
    e.release()


@pytest.mark.parametrize("spectrum", [eng.SPECTRUM_FP16, eng.SPECTRUM_BF16])
def test_engine_scaled_spectra_with_denormal_partitions_stay_finite(tan_ctx, spectrum):
    """IRs whose late partitions hold only denormal samples (a fast decay over
    a long IR): the per-partition power-of-two scale stays a normal number, so
    no partition turns into inf or NaN, and the output keeps its precision."""
    g = H.rng(20261203 + 51)
    B, nb, C, L = 256, 40, 2, 8192
    h = H.irs(g, C, L)
    h[:, 3 * B:5 * B] = (g.standard_normal((C, 2 * B)) * 1e-41).astype(np.float32)  # denormal partitions 3, 4
    h[:, 6 * B:] = 0.0
    x = H.noise(g, C, nb * B)
    sessions = [{"C": C, "L": L, "x": x, "events": {0: h}, "start": 0}]
    engine = eng.Engine(tan_ctx, B, spectrum, budget_bytes=64 << 20, max_channels=4)
    y = run_engine(engine, sessions, nb)[0]
    engine.release()
    assert np.isfinite(y).all()
    exp = fp64.stream_fp64(x, B, [(0, {c: h[c] for c in range(C)})])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < (-60 if spectrum == eng.SPECTRUM_FP16 else -40)


@pytest.mark.parametrize("B", [128, 512, 1024, 2048])
def test_engine_block_sizes_match_alone_and_fp64(tan_ctx, B):
    """Every block size the engine runs besides 256: sessions of one, two and
    eight partitions with IR swaps (on the first block, mid-stream, and on
    the block a later session opens) equal each session alone through the
    single-object path and the FP64 statement."""
    g = H.rng(20261204 + 60 + B)
    nb = 20
    specs = [(2, B, 0, [0, 9]), (1, 2 * B, 1, [0, 5]), (3, 7 * B + 5, 0, [0, 1, 13])]
    sessions = make_sessions(g, B, specs, nb)
    engine = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=16, partitions_per_item=2)
    outs = run_engine(engine, sessions, nb)
    engine.release()
    for s, y in zip(sessions, outs):
        ya = alone(tan_ctx, s["x"], B, s["events"])
        rms = np.sqrt(np.mean(ya.astype(np.float64) ** 2))
        assert np.max(np.abs(y - ya)) <= TOL * rms, (B, s["C"], s["L"])
        exp = fp64.stream_fp64(s["x"], B, [(k, {c: ir[c] for c in range(s["C"])}) for k, ir in s["events"].items()])
        for c in range(s["C"]):
            assert fp64.error_db(y[c], exp[c]) < -120, (B, s["L"], c)


@pytest.mark.parametrize("B", [256, 1024])
def test_engine_many_heads_same_bits(tan_ctx, B):
    """A launch with more heads than twice the SM count reads the twiddle table
    through L1 instead of copying it to shared memory: a session in it gives
    the samples it gives in a launch of few heads, bit for bit."""
    g = H.rng(20261204 + 70 + B)
    nb = 12
    test = make_sessions(g, B, [(2, 5000, 0, [0, 6])], nb)[0]
    crowd = make_sessions(g, B, [(8, 1000, 0, [0])] * 40, nb)  # 320 more channel slots
    big = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=400, partitions_per_item=8)
    y_big = run_engine(big, crowd + [test], nb)[-1]
    assert big.info()["slot_hwm"] > 2 * 148
    big.release()
    small = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 28, max_channels=8, partitions_per_item=8)
    y_small = run_engine(small, [test], nb)[0]
    small.release()
    assert np.array_equal(y_big, y_small)


@pytest.mark.parametrize("B", [128, 1024])
@pytest.mark.parametrize("spectrum,limit_db", [(eng.SPECTRUM_FP16, -60.0), (eng.SPECTRUM_BF16, -40.0),
                                               (eng.SPECTRUM_FP24, -90.0)])
def test_engine_reduced_precision_at_other_block_sizes(tan_ctx, B, spectrum, limit_db):
    """The 16- and 24-bit spectrum forms at the smallest and a large block
    size, with a swap mid-stream and a session of one partition: every
    channel within the form's bound of the FP64 statement."""
    g = H.rng(20261204 + 80 + B + spectrum)
    nb = 16
    specs = [(2, 9 * B + 7, 0, [0, 6]), (1, B, 1, [0])]
    sessions = make_sessions(g, B, specs, nb)
    engine = eng.Engine(tan_ctx, B, spectrum, budget_bytes=1 << 28, max_channels=16, partitions_per_item=4)
    outs = run_engine(engine, sessions, nb)
    engine.release()
    for s, y in zip(sessions, outs):
        exp = fp64.stream_fp64(s["x"], B, [(k, {c: ir[c] for c in range(s["C"])}) for k, ir in s["events"].items()])
        for c in range(s["C"]):
            assert fp64.error_db(y[c], exp[c]) < limit_db, (B, spectrum, s["L"], c)
