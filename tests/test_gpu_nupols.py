"""Non-uniformly partitioned convolution on the GPU against the FP64
statement: zero added latency, every schedule (doubling levels, single-partition
middle levels, uniform) gives the linear convolution; FP16 / BF16 spectra are
reported in dB. Tolerance for FP32: error < -120 dB of the output."""
import numpy as np
import pytest

from oracle import fp64
from tan_b200 import convolution as cv
from tan_b200 import nupols
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("C,L,levels,nb", [
    (2, 20000, [(64, 2), (128, 2), (256, 2), (512, 38)], 120),
    (3, 30000, [(128, 2), (256, 1), (512, 1), (1024, 1), (2048, 14)], 80),
    (1, 70000, [(128, 2), (256, 2), (512, 2), (1024, 2), (2048, 2), (4096, 2), (8192, 7)], 96),
    (2, 5000, [(256, 20)], 30),
])
def test_nu_matches_fp64(tan_ctx, C, L, levels, nb):
    g = H.rng(L + C)
    B = levels[0][0]
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L, (0.3, 1.0))
    nu = nupols.NonUniform(tan_ctx, C, L, levels)
    assert nu.set_response(h) == cv.AMF_OK, cv.last_error()
    y = nu.run(x)
    for c in range(C):
        assert fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) < -120
    nu.release()


def test_nu_default_schedule_long_ir_and_device_io(tan_ctx):
    import torch

    g = H.rng(77)
    C, L, B = 2, 1 << 17, 128
    levels = nupols.schedule(L, B, 4096)
    assert nupols.coverage(levels) >= L and levels[0] == (128, 2)
    nb = 300
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L, (1.0, 2.0))
    a = nupols.NonUniform(tan_ctx, C, L, levels)
    assert a.set_response(h) == 0
    y = a.run(x)
    for c in range(C):
        assert fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) < -120
    b = nupols.NonUniform(tan_ctx, C, L, levels)
    assert b.set_response(h) == 0
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    T = x.shape[1]
    for k in range(nb):
        assert b.process_device(xd.data_ptr() + k * B * 4, yd.data_ptr() + k * B * 4, T) == 0
    assert b.synchronize() == 0
    assert np.array_equal(yd.cpu().numpy(), y)
    a.release()
    b.release()


@pytest.mark.parametrize("spectrum,limit_db", [(1, -60.0), (2, -40.0)])
def test_nu_reduced_precision_db(tan_ctx, spectrum, limit_db):
    g = H.rng(88 + spectrum)
    C, L = 2, 40000
    levels = nupols.schedule(L, 128, 2048)
    nb = 150
    x = H.noise(g, C, nb * 128)
    h = H.irs(g, C, L, (0.5, 1.5))
    nu = nupols.NonUniform(tan_ctx, C, L, levels, spectrum)
    assert nu.set_response(h) == 0
    y = nu.run(x)
    worst = max(fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) for c in range(C))
    print(f"non-uniform spectrum {spectrum}: worst channel {worst:.1f} dB")
    assert worst < limit_db
    nu.release()


def test_nu_rejects_schedules_that_add_latency(tan_ctx):
    with pytest.raises(cv.TANError):
        nupols.NonUniform(tan_ctx, 1, 10000, [(128, 1), (256, 40)])  # level 1 starts at 128 < 256
    with pytest.raises(cv.TANError):
        nupols.NonUniform(tan_ctx, 1, 10000, [(128, 2), (256, 2)])  # does not cover the IR


@pytest.mark.parametrize("C,levels,nb", [
    (2, [(128, 2), (256, 1), (512, 1), (1024, 1), (2048, 1), (4096, 8)], 260),   # the 2^20-tap 256-channel schedule's shape, every level reached
    (2, [(128, 2), (256, 2), (512, 2), (1024, 2), (2048, 6)], 200),
    (64, [(128, 2), (256, 1), (512, 1), (1024, 5)], 64),
    (2, [(128, 2), (256, 1), (512, 1), (1024, 1), (2048, 1), (4096, 1), (8192, 4)], 400),
    # enough channels that the creation-time zero fills are still running when
    # the twiddle tables are uploaded
    (128, [(128, 2), (256, 1), (512, 1), (1024, 1), (2048, 1), (4096, 20)], 400),
])
def test_nu_signal_longer_than_every_level_offset(tan_ctx, C, levels, nb):
    """The output window reaches every level's contributions, with several
    blocks of each level (its tail included)."""
    g = H.rng(sum(b * k for b, k in levels) + C)
    L = nupols.coverage(levels)
    B = levels[0][0]
    assert nb * B > L // 2
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L, (2.0, 4.0))
    nu = nupols.NonUniform(tan_ctx, C, L, levels)
    assert nu.set_response(h) == 0
    y = nu.run(x)
    for c in (range(C) if C <= 8 else (0, C // 2, C - 1)):
        assert fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) < -120, c
    nu.release()


def test_nonuniform_fp16_with_denormal_partitions_stays_finite(tan_ctx):
    """The standalone non-uniform object with FP16 spectra on an IR whose
    later level partitions hold only denormal samples: finite output."""
    g = H.rng(20261203 + 52)
    C, L, B0, nb = 2, 8192, 128, 80
    levels = nupols.schedule(L, B0, 1024)
    h = H.irs(g, C, L)
    h[:, 3000:] = (g.standard_normal((C, L - 3000)) * 1e-41).astype(np.float32)
    x = H.noise(g, C, nb * B0)
    nu = nupols.NonUniform(tan_ctx, C, L, levels, 1)
    assert nu.set_response(h) == 0
    y = nu.run(x)
    nu.release()
    assert np.isfinite(y).all()
