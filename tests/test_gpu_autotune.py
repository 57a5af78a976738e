"""Autotuner on the GPU: every compiled tiling is measured (block time with
the tail overlapping its head, and the tail alone), the choice is the shortest
block time, and an object created through tuned() runs the chosen tiling and
matches the default tiling's output to 1e-5 of RMS."""
import numpy as np
import pytest

from tan_b200 import autotune
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu


def test_tune_picks_shortest_block_and_tuned_object_runs_it(tan_ctx):
    B, L, C = 256, 5000, 3
    e = autotune.tune(tan_ctx, B, L, C, write=False)
    assert len(e["all"]) >= 8
    assert e["block_us"] == min(r["block_us"] for r in e["all"])
    assert all(r["block_us"] > 0 and r["tail_us"] > 0 for r in e["all"])
    g = H.rng(71)
    x = H.noise(g, C, 12 * B)
    h = H.irs(g, C, L)
    ref = cv.TANConvolution(tan_ctx)
    assert ref.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    y0, _ = H.run_stream(ref, x, B, {0: (h, None)})
    conv = cv.TANConvolution(tan_ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, L, B, C) == 0
    rc, t = conv.tiling(e["index"])
    assert rc == 0 and list(t) == e["tiling"]
    y1, _ = H.run_stream(conv, x, B, {0: (h, None)})
    rms = np.sqrt(np.mean(y0.astype(np.float64) ** 2))
    assert np.max(np.abs(y1 - y0)) <= 1e-5 * rms
    ref.Release()
    conv.Release()
