"""Non-uniformly partitioned sessions in the batched engine: levels of growing
block size along the IR in the same graph launch per block as every other
session, with IR swaps (one-block crossfade, the new IR's output exact over the
full input history). Each session's output must equal the FP64 statement of
the stream (<= -120 dB with FP32 spectra) and the same session run alone
through the uniformly partitioned TANConvolution (<= 1e-5 x rms), also when it
shares the engine with uniform sessions; swaps are placed at the start, while
level outputs are still in flight, mid-period and on level-period boundaries."""
import numpy as np
import pytest

from oracle import fp64
from tan_b200 import convolution as cv
from tan_b200 import engine as eng
from tan_b200 import nupols
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def uniform_alone(ctx, x, B, events):
    C = x.shape[0]
    L = max(ir.shape[1] for ir in events.values())
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    y, codes = H.run_stream(conv, x, B, {k: (ir, None) for k, ir in events.items()})
    conv.Release()
    assert all(c == 0 for c in codes)
    return y


def expected(x, B, events):
    C = x.shape[0]
    return fp64.stream_fp64(x, B, [(k, {c: ir[c] for c in range(C)}) for k, ir in events.items()])


def run(engine, sessions, nb, device=False):
    """sessions: list of dict(C, L, levels or None, x, events); returns outputs."""
    import torch

    B = engine.block
    live = []
    for s in sessions:
        if s.get("levels"):
            rc, sess = engine.open_session_nu(s["C"], s["L"], s["levels"])
        else:
            rc, sess = engine.open_session(s["C"], s["L"])
        assert rc == 0, cv.last_error()
        live.append(sess)
    outs = [np.zeros((s["C"], nb * B), np.float32) for s in sessions]
    nslots = engine.info()["slot_hwm"]
    if device:
        xd = torch.zeros((nslots, nb * B), dtype=torch.float32, device="cuda")
        for s, sess in zip(sessions, live):
            xd[sess.slots] = torch.from_numpy(s["x"]).cuda()
        yd = torch.zeros_like(xd)
    for k in range(nb):
        for s, sess in zip(sessions, live):
            if k in s["events"]:
                assert sess.update_response_td(s["events"][k], block_until_ready=True) == 0, cv.last_error()
            if not device:
                engine.inp[sess.slots] = s["x"][:, k * B:(k + 1) * B]
        if device:
            assert engine.process_device(xd.data_ptr() + k * B * 4, yd.data_ptr() + k * B * 4, nb * B) == 0, \
                cv.last_error()
        else:
            assert engine.process() == 0, cv.last_error()
            for y, sess in zip(outs, live):
                y[:, k * B:(k + 1) * B] = engine.out[sess.slots]
    if device:
        assert engine.synchronize() == 0
        yh = yd.cpu().numpy()
        for y, sess in zip(outs, live):
            y[:] = yh[sess.slots]
    return outs


def make(g, C, L, B, nb, swaps, levels=None, rt60=(0.2, 1.5)):
    return {"C": C, "L": L, "levels": levels, "x": H.noise(g, C, nb * B),
            "events": {k: H.irs(g, C, L, rt60) for k in swaps}}


@pytest.mark.parametrize("swaps", [[0], [0, 5, 37, 63, 64, 100], [3, 47]])
def test_nu_session_matches_fp64_and_uniform(tan_ctx, swaps):
    """B = 128, IR 20000, levels 128x2, 256x2, 512x2, 1024x18 (period 8
    blocks): swaps at the first block, while level outputs are in flight (5),
    mid-period (37), on a period boundary where the largest level's head is due
    (63) and right after (64)."""
    g = H.rng(20261203 + 21 + len(swaps))
    B, nb, L = 128, 120, 20000
    levels = nupols.schedule(L, B, 1024)
    s = make(g, 2, L, B, nb, swaps, levels)
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=256 << 20, max_channels=8, partitions_per_item=8)
    y = run(e, [s], nb)[0]
    e.release()
    exp = expected(s["x"], B, s["events"])
    for c in range(s["C"]):
        assert fp64.error_db(y[c], exp[c]) < -120, (c, fp64.error_db(y[c], exp[c]))
    ya = uniform_alone(tan_ctx, s["x"], B, s["events"])
    assert H.rel_err(y, ya) <= TOL


def test_nu_beside_uniform_sessions_mix_equals_alone(tan_ctx):
    """Two non-uniform sessions (different schedules) and two uniform ones in one
    engine, swaps at different blocks: each non-uniform session equals itself
    alone in its own engine bit for bit, and every session equals the uniform
    drop-in alone within tolerance."""
    g = H.rng(20261203 + 22)
    B, nb = 256, 96
    specs = [make(g, 2, 30000, B, nb, [0, 29], nupols.schedule(30000, B, 2048)),
             make(g, 1, 9000, B, nb, [0, 50]),
             make(g, 3, 65536, B, nb, [0, 15, 64], [(256, 4), (1024, 3), (4096, 15)]),
             make(g, 2, 4000, B, nb, [0])]
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=16)
    outs = run(e, specs, nb)
    e.release()
    for i, (s, y) in enumerate(zip(specs, outs)):
        ya = uniform_alone(tan_ctx, s["x"], B, s["events"])
        assert H.rel_err(y, ya) <= TOL, (i, H.rel_err(y, ya))
        if s["levels"]:
            solo = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 28, max_channels=4)
            ys = run(solo, [s], nb)[0]
            solo.release()
            assert np.array_equal(y, ys), i


def test_nu_device_io_equals_host_io(tan_ctx):
    """The host-buffer graph and direct launches with device rows run the same
    kernels: outputs are bit-identical, swaps included."""
    g = H.rng(20261203 + 23)
    B, nb = 128, 80
    specs = [make(g, 2, 12000, B, nb, [0, 31], nupols.schedule(12000, B, 1024)), make(g, 1, 3000, B, nb, [0, 9])]
    outs = []
    for device in (False, True):
        e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=256 << 20, max_channels=8)
        outs.append(run(e, specs, nb, device=device))
        e.release()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_nu_long_ir_up_to_16384_blocks(tan_ctx):
    """IR 2^20 at base block 128 with levels doubling to 16384 (the
    non-uniform benchmark's schedule), two channels over 640 blocks (the
    16384-sample level's first outputs land at tap 32512 and it runs 5 periods),
    swaps at 200 and 451."""
    g = H.rng(20261203 + 24)
    B, nb, L = 128, 640, 1 << 20
    levels = nupols.schedule(L, B, 16384)
    assert levels[-1][0] == 16384
    s = make(g, 2, L, B, nb, [0, 200, 451], levels, rt60=(8.0, 8.0))
    e = eng.Engine(tan_ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=4)
    y = run(e, [s], nb)[0]
    e.release()
    exp = expected(s["x"], B, s["events"])
    for c in range(s["C"]):
        assert fp64.error_db(y[c], exp[c]) < -120, (c, fp64.error_db(y[c], exp[c]))


@pytest.mark.parametrize("spectrum,limit_db", [(eng.SPECTRUM_FP16, -60.0), (eng.SPECTRUM_BF16, -40.0),
                                               (eng.SPECTRUM_FP24, -90.0)])
def test_nu_reduced_precision_error_db(tan_ctx, spectrum, limit_db):
    g = H.rng(20261203 + 25 + spectrum)
    B, nb, L = 128, 100, 40000
    s = make(g, 2, L, B, nb, [0, 41], nupols.schedule(L, B, 2048))
    e = eng.Engine(tan_ctx, B, spectrum, budget_bytes=256 << 20, max_channels=4)
    y = run(e, [s], nb)[0]
    e.release()
    exp = expected(s["x"], B, s["events"])
    worst = max(fp64.error_db(y[c], exp[c]) for c in range(s["C"]))
    print(f"spectrum {spectrum}: non-uniform worst channel error vs FP64 {worst:.1f} dB")
    assert worst < limit_db


def test_nu_schedule_checks(tan_ctx):
    e = eng.Engine(tan_ctx, 256, eng.SPECTRUM_FP32, budget_bytes=64 << 20, max_channels=4)
    assert e.open_session_nu(1, 10000, [(128, 2), (256, 40)])[0] == cv.AMF_INVALID_ARG  # level 0 != block
    assert e.open_session_nu(1, 10000, [(256, 1), (512, 20)])[0] == cv.AMF_INVALID_ARG  # starts before its block
    assert e.open_session_nu(1, 10000, [(256, 2), (512, 2), (384, 30)])[0] == cv.AMF_INVALID_ARG  # not a power of 2
    assert e.open_session_nu(1, 100000, [(256, 2), (512, 20)])[0] == cv.AMF_INVALID_ARG  # does not cover the IR
    assert e.open_session_nu(1, 1 << 22, [(256, 2), (512, 2), (32768, 128)])[0] == cv.AMF_INVALID_ARG  # > 16384
    rc, s = e.open_session_nu(1, 10000, [(256, 2), (512, 2), (1024, 9)])
    assert rc == 0 and s.close() == 0
    e.release()
