"""TANConverter / TANMixer on the GPU against the oracle's restatement, bit for
bit: host overloads follow the reference's CPU code (ConverterImpl.cpp,
MixerImpl.cpp), device overloads its OpenCL kernels (Converter.cl, Mixer.cl).
Covers strided (interleaved) buffers, ties, NaN, values beyond int range, the
clip report, batches of more buffers than one launch carries, and errors."""
import numpy as np
import pytest

from oracle import ref
from tan_b200 import convolution as cv
from tan_b200 import converter as cvt

pytestmark = pytest.mark.gpu


def _signal(g, n):
    x = g.uniform(-1.2, 1.2, n).astype(np.float32)
    x[::97] = 0.5 / 32767 * g.integers(-3, 4, x[::97].size)
    x[5::211] = np.float32(np.nan)
    x[7::223] = np.float32(1e6)
    x[9::229] = np.float32(-1e6)
    return x


@pytest.fixture(scope="module")
def conv_(tan_ctx):
    c = cvt.TANConverter(tan_ctx)
    yield c
    c.Terminate()


@pytest.mark.parametrize("n", [1, 7, 8, 13, 1000, 4099])
@pytest.mark.parametrize("gain", [1.0, 0.37])
def test_float_to_short_host_matches_cpu_reference(conv_, n, gain):
    g = np.random.Generator(np.random.PCG64(n))
    x = _signal(g, 2 * n)  # read with step 2
    y = np.full(3 * n, 1234, np.int16)  # written with step 3: other samples stay
    rc, clip = conv_.ConvertFloatToShort(x, 2, n, y, 3, gain)
    assert rc == 0
    ey, eclip = ref.convert_f32_s16(x, gain, in_step=2, n=n)
    assert np.array_equal(y[::3], ey) and clip == eclip
    assert np.all(y[1::3] == 1234) and np.all(y[2::3] == 1234)


def test_short_to_float_host(conv_):
    g = np.random.Generator(np.random.PCG64(1))
    x = g.integers(-32768, 32768, 3000).astype(np.int16)
    y = np.zeros(1500, np.float32)
    assert conv_.ConvertShortToFloat(x, 2, 1500, y, 1, 0.8) == 0
    assert np.array_equal(y, ref.convert_s16_f32(x, 0.8, in_step=2, n=1500))


def test_batches_host(conv_):
    g = np.random.Generator(np.random.PCG64(2))
    xs = [_signal(g, 523) for _ in range(70)]  # more buffers than one launch carries
    ys = [np.zeros(523, np.int16) for _ in range(70)]
    rc, clip = conv_.ConvertFloatToShortBatch(xs, 1, 523, ys, 1, 1.0)
    assert rc == 0
    exp = [ref.convert_f32_s16(x, 1.0) for x in xs]
    assert all(np.array_equal(y, e[0]) for y, e in zip(ys, exp))
    assert clip == any(e[1] for e in exp)
    si = [g.integers(-32768, 32768, 523).astype(np.int16) for _ in range(3)]
    so = [np.zeros(523, np.float32) for _ in range(3)]
    assert conv_.ConvertShortToFloatBatch(si, 1, 523, so, 1, 2.0) == 0
    assert all(np.array_equal(o, ref.convert_s16_f32(i, 2.0)) for i, o in zip(si, so))


def test_device_overloads_match_opencl_rules(conv_):
    import torch

    g = np.random.Generator(np.random.PCG64(3))
    x = _signal(g, 4000)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((2 * 2000 + 1,), 77, dtype=torch.int16, device="cuda")
    # float -> short, step 2 with offsets (interleaved stereo, right channel)
    rc, clip = conv_.ConvertDevice([xd], 2, [1], cvt.TAN_SAMPLE_TYPE_FLOAT, [yd], 2, [1], cvt.TAN_SAMPLE_TYPE_SHORT,
                                   1999, 1.0, want_clipped=True)
    assert rc == 0
    ey, eclip = ref.convert_f32_s16(x[1:], 1.0, in_step=2, n=1999, device=True)
    y = yd.cpu().numpy()
    assert np.array_equal(y[1:2 * 1999:2], ey) and clip == eclip
    assert np.all(y[0::2] == 77)
    # short -> float and the two copies
    s = torch.from_numpy(g.integers(-32768, 32768, 1000).astype(np.int16)).cuda()
    f = torch.zeros(1000, device="cuda")
    rc, _ = conv_.ConvertDevice([s], 1, None, cvt.TAN_SAMPLE_TYPE_SHORT, [f], 1, None, cvt.TAN_SAMPLE_TYPE_FLOAT,
                                1000, 0.5)
    assert rc == 0 and conv_.Synchronize() == 0
    assert np.array_equal(f.cpu().numpy(), ref.convert_s16_f32(s.cpu().numpy(), 0.5))
    s2 = torch.zeros_like(s)
    assert conv_.ConvertDevice([s], 1, None, 1, [s2], 1, None, 1, 1000, 1.0)[0] == 0
    f2 = torch.zeros_like(f)
    assert conv_.ConvertDevice([f], 1, None, 0, [f2], 1, None, 0, 1000, 1.0)[0] == 0
    conv_.Synchronize()
    assert torch.equal(s, s2) and torch.equal(f, f2)


def test_converter_errors(conv_):
    x = np.zeros(8, np.float32)
    y = np.zeros(8, np.int16)
    assert conv_.ConvertFloatToShort(x, 1, 0, y, 1, 1.0)[0] == cv.AMF_INVALID_ARG
    assert conv_.ConvertFloatToShort(x, 1, 8, y, 1, 0.0)[0] == cv.AMF_INVALID_ARG
    assert cv.lib().tanb_converter_convert_device(conv_._h, None, 1, None, 0, None, 1, None, 1, 8, 1.0, 1,
                                                  None) == cv.AMF_INVALID_ARG
    import torch

    xd = torch.zeros(8, device="cuda")
    yd = torch.zeros(8, dtype=torch.int16, device="cuda")
    assert conv_.ConvertDevice([xd], 1, None, 0, [yd], 1, None, 1, 8, 1.0)[0] == 0
    assert conv_.ConvertDevice([xd], 1, None, 0, [yd], 1, None, 7, 8, 1.0)[0] == cv.AMF_NOT_IMPLEMENTED


@pytest.mark.parametrize("channels", [1, 5, 70])
def test_mixer(tan_ctx, channels):
    import torch

    g = np.random.Generator(np.random.PCG64(channels))
    n = 1029
    x = g.standard_normal((channels, n)).astype(np.float32)
    x[0, 3] = -0.0
    m = cvt.TANMixer(tan_ctx, n, channels)
    y = np.zeros(n, np.float32)
    assert m.Mix([x[c] for c in range(channels)], y) == 0
    e = ref.mix(x)
    assert np.array_equal(y.view(np.uint32), e.view(np.uint32))  # signed zero included
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(n, device="cuda")
    assert m.MixDevice([xd[c] for c in range(channels)], yd) == 0
    m.Synchronize()
    ed = ref.mix(x, device=True)
    assert np.array_equal(yd.cpu().numpy().view(np.uint32), ed.view(np.uint32))
    wide = torch.zeros((channels, n + 11), device="cuda")
    wide[:, :n] = xd
    yd2 = torch.zeros(n, device="cuda")
    assert m.MixDeviceStrided(wide, yd2, n + 11) == 0
    m.Synchronize()
    assert np.array_equal(yd2.cpu().numpy().view(np.uint32), ed.view(np.uint32))
    m.Terminate()
