"""The oracle's restatement of the room response producer (GPU path of
TrueAudioVR::generateRoomResponse): image counts follow the reference's grid
(2n per axis rounded up to the local size 4, ids above 2n idle), the direct
sound arrives at 1 + (int)(d / 340 * rate), bounce limits shrink the grid,
and a listener facing the source symmetrically hears mirrored ears."""
import numpy as np

from oracle import ref

ROOM = (8.0, 3.0, 6.0, 0.3, 0.3, 0.5, 0.5, 0.4, 0.4)


def _extent(n2):
    return min(n2 + (4 - n2 % 4) % 4, n2 + 1)


def test_image_count_and_direct_arrival():
    lp, hp = ref.simple_head_filters()
    rate, length = 48000, 24000
    left, right, n = ref.room_response(ROOM, (2.0, 1.5, 1.0), (4.0, 1.5, 4.0, 0.16, 0.0, 0.0, 0.0), rate, length,
                                       lp, hp)
    nsw, nsh, nsl = (int(np.float32(s) / np.float32(340.0) * rate) for s in ROOM[:3])
    nW, nH, nL = 1 + length // nsw, 1 + length // nsh, 1 + length // nsl
    assert n == _extent(2 * nW) * _extent(2 * nH) * _extent(2 * nL)
    # direct path to the left ear (offset +spacing/2 along x without rotation)
    d = np.sqrt(np.float32((2.0 - 4.08) ** 2 + 0.0 + (1.0 - 4.0) ** 2))
    first = 1 + int(d / 340.0 * rate)
    nz = np.nonzero(left)[0]
    assert abs(nz[0] - first) <= 1 and np.abs(left[:first - 1]).max() == 0
    assert np.isfinite(left).all() and np.isfinite(right).all()


def test_bounce_limit_and_mirror_symmetry():
    lp, hp = ref.simple_head_filters()
    full = ref.room_response(ROOM, (4.0, 1.5, 1.0), (4.0, 1.5, 4.0, 0.16, 0.0, 0.0, 0.0), 48000, 12000, lp, hp)
    lim = ref.room_response(ROOM, (4.0, 1.5, 1.0), (4.0, 1.5, 4.0, 0.16, 0.0, 0.0, 0.0), 48000, 12000, lp, hp,
                            flags=0x40, max_bounces=2)
    assert lim[2] == _extent(4) ** 3 and lim[2] < full[2]
    # source on the listener's median plane, symmetric walls: the two ears
    # see mirrored geometry, so their direct arrivals coincide
    l, r = full[0], full[1]
    assert np.nonzero(l)[0][0] == np.nonzero(r)[0][0]
    assert abs(np.sum(l[:2000]) - np.sum(r[:2000])) < 1e-3 * np.sum(np.abs(l[:2000]))
