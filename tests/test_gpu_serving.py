"""The serving loop (tan_b200.serving.serve) at small scale on the GPU:
Poisson arrivals admitted by the device-memory budget, exponential lifetimes,
IR swaps, one engine block per block period with a control thread uploading
IRs and closing sessions beside it. Sessions traced by the loop (their swaps on
known blocks) must equal the same session alone through TANConvolution
(<= 1e-5 x rms), in the mix with every other session coming and going."""
import numpy as np
import pytest

from tan_b200 import convolution as cv
from tan_b200 import engine as eng
from tan_b200 import serving
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def alone(ctx, x, B, events):
    C = x.shape[0]
    L = max(ir.shape[1] for ir in events.values())
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    y, codes = H.run_stream(conv, x, B, {k: (ir, None) for k, ir in events.items()})
    conv.Release()
    assert all(c == 0 for c in codes)
    return y


@pytest.mark.parametrize("spectrum", [eng.SPECTRUM_FP32])
def test_serve_loop_admits_churns_and_traced_sessions_match_alone(tan_ctx, spectrum):
    B = 256
    r = serving.serve(tan_ctx, seconds=1.5, rate=30.0, lifetime=0.4, swap_rate=6.0, block=B, spectrum=spectrum,
                      budget=96 << 20, max_channels=512, ch_range=(1, 3), len_range=(4096, 30000),
                      prefill=False, trace=3)
    assert r["blocks"] == int(1.5 * 48000 / B)
    assert r["admitted"] >= 10 and not r["control_errors"], r
    assert r["latency_ms"]["p50"] < r["deadline_ms"]
    assert r["concurrent_channels_max"] >= 3
    assert len(r["traces"]) == 3
    for tr in r["traces"]:
        y = tr["y"]
        nb = y.shape[1] // B
        assert nb > 20 and len(tr["events"]) >= 2  # the loop swapped its IR at least once
        x = np.tile(tr["x"], (1, nb))
        assert H.rel_err(y, alone(tan_ctx, x, B, tr["events"])) <= TOL
