"""Default non-uniform level schedule (tanb_nu_schedule, host code, no GPU):
block sizes are powers of two that start at the base block and double, two
partitions per size until the largest size, which covers the rest of the IR;
the levels together cover the IR; each level's first tap is at or after its
block size (zero added latency); invalid arguments are rejected."""
import pytest

from tan_b200 import nupols
from tan_b200.convolution import TANError


@pytest.mark.parametrize("L,B0,Nmax", [(1 << 20, 128, 8192), (48000, 256, 4096), (100, 128, 1024),
                                       (65536, 512, 512), (300000, 32, 8192), (1 << 20, 128, 16384)])
def test_schedule_shape_and_coverage(L, B0, Nmax):
    levels = nupols.schedule(L, B0, Nmax)
    assert 1 <= len(levels) <= 16
    blocks = [b for b, _ in levels]
    assert blocks[0] == B0
    assert all(b & (b - 1) == 0 and B0 <= b <= Nmax for b in blocks)
    assert all(blocks[i + 1] in (blocks[i], 2 * blocks[i]) for i in range(len(blocks) - 1))
    assert all(k == 2 for _, k in levels[:-1])
    assert nupols.coverage(levels) >= L
    assert nupols.coverage(levels[:-1]) < L
    off = 0
    for i, (b, k) in enumerate(levels):
        if i:
            assert off >= b, (i, off, b)  # the level's first tap is at or after its block
        off += b * k


@pytest.mark.parametrize("args", [(1000, 100, 1024), (1000, 256, 128), (1000, 16, 1024), (1000, 128, 32768),
                                  (0, 128, 1024)])
def test_schedule_rejects_invalid_arguments(args):
    with pytest.raises(TANError):
        nupols.schedule(*args)
