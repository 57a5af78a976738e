"""GPU room response producer against the oracle's restatement, bit for bit
(exact 64-bit fixed-point sums and explicit IEEE operations on both sides),
and end to end: IRs generated in device memory, handed to
UpdateResponseTDDevice, give the same convolution output as the oracle's IRs
uploaded from the host."""
import numpy as np
import pytest

from oracle import ref
from tan_b200 import convolution as cv
from tan_b200 import roomgen as rg
from tests import helpers as H

pytestmark = pytest.mark.gpu

CASES = [
    # room (w, h, l, damp L R T B F Bk), source, ears (x, y, z, spacing, yaw, pitch, roll), rate, length, flags, max
    ((8.0, 3.0, 6.0, 0.3, 0.3, 0.5, 0.5, 0.4, 0.4), (2.0, 1.5, 1.0), (4.0, 1.6, 4.0, 0.16, 30.0, 0.0, 0.0),
     48000, 48000, 0, 0),
    ((5.0, 2.5, 4.0, 0.6, 0.2, 0.7, 0.1, 0.5, 0.3), (9.0, -1.0, 2.0), (2.5, 1.2, 1.0, 0.18, -45.0, 10.0, 5.0),
     44100, 30001, 0, 0),
    ((20.0, 6.0, 12.0, 0.2, 0.25, 0.3, 0.35, 0.4, 0.45), (3.0, 2.0, 9.0), (12.0, 1.7, 3.0, 0.15, 90.0, -20.0, 0.0),
     48000, 65536, rg.GENROOM_LIMIT_BOUNCES, 6),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_room_response_matches_oracle(tan_ctx, case):
    import torch

    room, src, ears, rate, length, flags, mb = CASES[case]
    lp, hp = ref.simple_head_filters(ear_spacing=ears[3])
    el, er, n = ref.room_response(room, src, ears, rate, length, lp, hp, flags, mb)
    gen = rg.RoomGenerator(tan_ctx, 70000)
    L = rg.listener(ears[:3], ears[3], *ears[4:], lp, hp)
    left = torch.full((length,), 7.0, device="cuda")
    right = torch.full((length,), 7.0, device="cuda")
    for _ in range(2):  # twice: the accumulator must be clear again after a call
        assert gen.response(rg.Room(*room), rg.Source(*src), L, rate, length, left, right, flags, mb) == 0, \
            cv.last_error()
        assert gen.synchronize() == 0
        assert gen.images() == n
        assert np.array_equal(left.cpu().numpy(), el) and np.array_equal(right.cpu().numpy(), er)
    # on a caller's stream
    s = torch.cuda.Stream()
    left2 = torch.zeros(length, device="cuda")
    right2 = torch.zeros(length, device="cuda")
    assert gen.response(rg.Room(*room), rg.Source(*src), L, rate, length, left2, right2, flags, mb,
                        stream=s.cuda_stream) == 0
    s.synchronize()
    assert torch.equal(left2, left) and torch.equal(right2, right)
    gen.release()


def test_room_response_errors(tan_ctx):
    import torch

    gen = rg.RoomGenerator(tan_ctx, 1000)
    lp, hp = ref.simple_head_filters()
    L = rg.listener((1.0, 1.0, 1.0), 0.16, 0.0, 0.0, 0.0, lp, hp)
    buf = torch.zeros(2000, device="cuda")
    room = rg.Room(4.0, 3.0, 4.0, 0.5, 0.5, 0.5, 0.5, 0.5, 0.5)
    assert gen.response(room, rg.Source(1, 1, 1), L, 48000, 1001, buf, buf) == cv.AMF_INVALID_ARG
    assert gen.response(room, rg.Source(1, 1, 1), L, 48000, 500, buf, buf, rg.GENROOM_LIMIT_BOUNCES, 0) == \
        cv.AMF_INVALID_ARG
    tiny = rg.Room(0.001, 3.0, 4.0, 0.5, 0.5, 0.5, 0.5, 0.5, 0.5)
    assert gen.response(tiny, rg.Source(0, 1, 1), L, 48000, 500, buf, buf) == cv.AMF_INVALID_ARG
    gen.release()


def test_generated_irs_feed_update_on_device(tan_ctx):
    """The sample's pattern (SimpleVRaudio.cpp:914-925): regenerate the room
    response for a moved listener and swap it in without a host round trip."""
    import torch

    room, src, ears, rate, _, _, _ = CASES[0]
    B, length, nb = 256, 20000, 24
    lp, hp = ref.simple_head_filters()
    gen = rg.RoomGenerator(tan_ctx, length)
    dev = cv.TANConvolution(tan_ctx)
    assert dev.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, length, B, 2) == 0
    host = cv.TANConvolution(tan_ctx)
    assert host.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, length, B, 2) == 0
    g = H.rng(5)
    x = H.noise(g, 2, nb * B)
    irs = torch.zeros((2, 2, length), device="cuda")
    events = {}
    for j, (k, yaw) in enumerate(((0, 0.0), (11, 40.0))):
        L = rg.listener(ears[:3], ears[3], yaw, 0.0, 0.0, lp, hp)
        assert gen.response(rg.Room(*room), rg.Source(*src), L, rate, length, irs[j, 0], irs[j, 1],
                            stream=dev.stream()) == 0
        el, er, _ = ref.room_response(room, src, ears[:4] + (yaw, 0.0, 0.0), rate, length, lp, hp)
        events[k] = (j, np.stack([el, er]))
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    for k in range(nb):
        if k in events:
            j = events[k][0]
            assert dev.UpdateResponseTDDevice([irs[j, 0], irs[j, 1]], length) == 0
        rc, done = dev.ProcessDevice([xd[c, k * B:(k + 1) * B] for c in range(2)],
                                     [yd[c, k * B:(k + 1) * B] for c in range(2)], B)
        assert rc == 0 and done == B
    assert dev.Synchronize() == 0
    y_host, _ = H.run_stream(host, x, B, {k: (ir, None) for k, (_, ir) in events.items()})
    assert np.array_equal(yd.cpu().numpy(), y_host)
    gen.release()
    dev.Release()
    host.Release()
