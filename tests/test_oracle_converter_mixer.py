"""The oracle's restatement of TANConverter / TANMixer (oracle/tan_cpu_ref.cpp)
against an independent numpy statement of the reference's rules:
ConverterImpl.cpp:217-408 (CPU overloads), Converter.cl:97-120 and
Mixer.cl:26-41 (device overloads), MixerImpl.cpp:226-250. No reference test
or fixture covers these components, so this pins the restatement to the
reference source's arithmetic, operation by operation."""
import numpy as np
import pytest

from oracle import ref

INT_MIN = -2 ** 31


def _rne_sse(f):
    """cvtps2dq: round half to even; NaN and |f| >= 2^31 give INT_MIN."""
    out = np.full(f.shape, INT_MIN, np.int64)
    ok = np.isfinite(f) & (f < 2.0 ** 31) & (f >= -2.0 ** 31)
    out[ok] = np.rint(f[ok].astype(np.float64)).astype(np.int64)
    return out


def _trunc_sse(f):
    out = np.full(f.shape, INT_MIN, np.int64)
    ok = np.isfinite(f) & (f < 2.0 ** 31) & (f >= -2.0 ** 31)
    out[ok] = np.trunc(f[ok].astype(np.float64)).astype(np.int64)
    return out


def _expected_cpu(x, gain):
    scale = np.float32(32767) * np.float32(gain)
    f = (x.astype(np.float32) * scale).astype(np.float32)
    n8 = (x.size // 8) * 8
    y = np.empty(x.size, np.int64)
    y[:n8] = np.clip(_rne_sse(f[:n8]), -32768, 32767)
    t = _trunc_sse(f[n8:])
    clip = bool(np.any((t > 32767) | (t < -32768)))
    y[n8:] = np.clip(t, -32768, 32767)
    return y.astype(np.int16), clip


def _expected_dev(x, gain):
    scale = np.float32(32767) * np.float32(gain)
    f = (x.astype(np.float32) * scale).astype(np.float32)
    clip = bool(np.any(f > 32767) | np.any(f < -32768))
    g = np.clip(f, -32768, 32767)
    g = np.where(np.isnan(g), 0, g)
    return np.trunc(g).astype(np.int16), clip


def _signal(g, n):
    x = g.uniform(-1.2, 1.2, n).astype(np.float32)
    x[::97] = 0.5 / 32767 * g.integers(-3, 4, x[::97].size)  # exact .5 ties after scaling
    x[5::211] = np.float32(np.nan)
    x[7::223] = np.float32(1e6)   # product beyond 2^31
    x[9::229] = -np.float32(-1e6)
    return x


@pytest.mark.parametrize("n", [1, 7, 8, 13, 64, 1000, 4099])
@pytest.mark.parametrize("gain", [1.0, 0.37, 2.5])
def test_float_to_short_cpu_overload(n, gain):
    g = np.random.Generator(np.random.PCG64(n))
    x = _signal(g, n)
    y, clip = ref.convert_f32_s16(x, gain)
    ey, eclip = _expected_cpu(x, gain)
    assert np.array_equal(y, ey)
    assert clip == eclip


@pytest.mark.parametrize("n", [1, 9, 1000])
def test_float_to_short_device_rules(n):
    g = np.random.Generator(np.random.PCG64(100 + n))
    x = _signal(g, n)
    y, clip = ref.convert_f32_s16(x, 1.0, device=True)
    ey, eclip = _expected_dev(x, 1.0)
    assert np.array_equal(y, ey) and clip == eclip


def test_float_to_short_strided_and_clip_only_in_tail():
    # interleaved stereo as in the samples (step 2); a clipped sample inside a
    # full group of 8 is saturated but not reported by the CPU overload
    x = np.zeros(2 * 16, np.float32)
    x[2 * 3] = 2.0
    y, clip = ref.convert_f32_s16(x, 1.0, in_step=2, n=16)
    assert y[3] == 32767 and not clip
    x[2 * 15] = -3.0
    y, clip = ref.convert_f32_s16(x, 1.0, in_step=2, n=16)
    assert y[15] == -32768 and not clip   # 16 samples: two full groups
    # n = 12: samples 8..11 are the tail; a clamped sample there is reported
    x2 = np.zeros(2 * 12, np.float32)
    x2[2 * 10] = -3.0
    y, clip = ref.convert_f32_s16(x2, 1.0, in_step=2, n=12)
    assert y[10] == -32768 and clip


def test_short_to_float():
    g = np.random.Generator(np.random.PCG64(3))
    x = g.integers(-32768, 32768, 5000).astype(np.int16)
    for gain in (1.0, 0.25, 3.0):
        y = ref.convert_s16_f32(x, gain)
        assert np.array_equal(y, x.astype(np.float32) * np.float32(np.float32(gain) / np.float32(32767)))
    y = ref.convert_s16_f32(x, 1.0, in_step=3)
    assert np.array_equal(y, x[::3].astype(np.float32) * np.float32(1.0 / 32767))


def test_mix_orders():
    g = np.random.Generator(np.random.PCG64(4))
    x = g.standard_normal((7, 513)).astype(np.float32)
    x[0, 0] = -0.0
    exp = x[0].copy()
    for c in range(1, 7):
        exp = (exp + x[c]).astype(np.float32)
    y = ref.mix(x)
    assert np.array_equal(y, exp) and np.signbit(y[0]) == np.signbit(exp[0])
    yd = ref.mix(x, device=True)
    expd = np.zeros(513, np.float32)
    for c in range(7):
        expd = (expd + x[c]).astype(np.float32)
    assert np.array_equal(yd, expd)
