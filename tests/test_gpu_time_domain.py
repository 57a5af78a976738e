"""TIME_DOMAIN method on the GPU: ProcessDirect against the oracle's restatement
of ovlTimeDomainCPU (ConvolutionImpl.cpp:2757-2782) and Process with IR swaps
against the FP64 statement. Tolerance: 1e-5 x rms of the expected output."""
import numpy as np
import pytest

from oracle import fp64, ref
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu


def make(ctx, L, B, C):
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_TIME_DOMAIN, L, B, C) == cv.AMF_OK, cv.last_error()
    return conv


@pytest.mark.parametrize("L,calls", [(300, [200, 200, 57, 256, 1, 300]), (4096, [4096, 1000, 3000]),
                                     (2000, [64, 2048, 2048, 7])])
def test_process_direct_matches_restatement(tan_ctx, L, calls):
    g = H.rng(L)
    C = 3
    length = 1 << (L - 1).bit_length()
    gpu = make(tan_ctx, L, 128, C)
    oracle = ref.RefTimeDomain(L, C)
    for i, n in enumerate(calls):
        ir = np.zeros((C, length), np.float32)
        ir[:, :L] = H.irs(g, C, L)
        x = H.noise(g, C, n)
        nz = None
        if i % 2 == 1:
            nz = np.array([[3, L - 5], [0, L], [L // 2, L // 2 + 17]], np.int32).reshape(-1)
        y = np.zeros_like(x)
        rc, done = gpu.ProcessDirect(ir, x, y, n, nz)
        assert rc == 0 and done == min(n, length), (rc, cv.last_error())
        rcr, yr, doner = oracle.process_direct(ir, x, nz)
        assert rcr == 0 and doner == done
        scale = np.sqrt(np.mean(yr.astype(np.float64) ** 2)) + 1e-30
        assert np.max(np.abs(y - yr)) <= 1e-5 * scale


def test_process_direct_is_fp64_convolution_when_history_fits(tan_ctx):
    """n + L - 1 <= nextpow2(L): the circular history holds every tap's input."""
    g = H.rng(2)
    C, L, n = 2, 900, 120  # nextpow2 = 1024 >= 900 + 120 - 1
    gpu = make(tan_ctx, L, 128, C)
    h = np.zeros((C, 1024), np.float32)
    h[:, :L] = H.irs(g, C, L)
    x = H.noise(g, C, n * 20)
    y = np.zeros_like(x)
    for k in range(20):
        ys = np.zeros((C, n), np.float32)
        rc, done = gpu.ProcessDirect(h, np.ascontiguousarray(x[:, k * n:(k + 1) * n]), ys, n)
        assert rc == 0 and done == n
        y[:, k * n:(k + 1) * n] = ys
    for c in range(C):
        assert fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) < -120


def test_time_domain_process_with_swaps(tan_ctx):
    g = H.rng(3)
    C, L, B, nb = 2, 900, 64, 40  # B + L - 1 <= 1024
    gpu = make(tan_ctx, L, B, C)
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    y, codes = H.run_stream(gpu, x, B, {0: (h0, None), 17: (h1, None)})
    assert all(c == 0 for c in codes)
    exp = fp64.stream_fp64(x, B, [(0, {c: h0[c] for c in range(C)}), (17, {c: h1[c] for c in range(C)})])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120


def test_time_domain_errors(tan_ctx):
    gpu = make(tan_ctx, 256, 64, 2)
    x = np.zeros((2, 64), np.float32)
    bad = np.array([0, 300, 0, 10], np.int32)  # last beyond the history length
    rc, _ = gpu.ProcessDirect(np.zeros((2, 256), np.float32), x, x.copy(), 64, bad)
    assert rc == cv.AMF_INVALID_ARG
    fft = cv.TANConvolution(tan_ctx)
    assert fft.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, 256, 64, 2) == 0
    rc, _ = fft.ProcessDirect(np.zeros((2, 256), np.float32), x, x.copy(), 64)
    assert rc == cv.AMF_NOT_SUPPORTED
    gpu.Release()
    fft.Release()
