"""GPU test of tanb_convolve_no_alloc, the entry point for callers that cannot
allocate device memory (it keeps its temporaries in a fixed library-owned
array). Its output is checked against the existing TANConvolution path
(Init + UpdateResponseTD + Process through the C ABI) on the same inputs, on
calls in a row, within the parity tolerance of the other GPU tests
(1e-5 x rms), and against the FP64 statement of the convolution (-120 dB). The object path crossfades block 0 from its initial zero IR, so
that block is compared against the no-alloc output times the crossfade ramp.
This file is collected last so a run that stops at the first failure has
already run every other test."""
import numpy as np
import pytest

from oracle import fp64
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _object_path(ctx, x, h, B):
    C, T = x.shape
    conv = cv.TANConvolution(ctx)
    assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM, h.shape[1], B, C) == cv.AMF_OK
    assert conv.UpdateResponseTD(h, h.shape[1]) == cv.AMF_OK
    y = np.zeros_like(x)
    rc, done = conv.Process(x, y, T)
    assert rc == cv.AMF_OK and done == T
    conv.Release()
    return y


def test_no_alloc_matches_object_path_on_two_calls():
    """Calls in a row with different shapes: many partitions, one partition
    (ir_length <= block: the head alone), two partitions (no tail launch), and
    one call on a side stream. Each output is checked against the object path
    and against the FP64 statement of the convolution."""
    import torch

    ctx = cv.TANContext(0)
    lib = cv.lib()
    side = torch.cuda.Stream()
    cases = [(3, 256, 3000, 12, False), (2, 512, 9000, 10, False), (2, 256, 200, 6, False),
             (2, 256, 400, 7, True)]
    for call, (C, B, L, nb, on_side) in enumerate(cases):
        g = H.rng(4242 + call)
        x = H.noise(g, C, nb * B)
        h = H.irs(g, C, L)
        xd = torch.from_numpy(x).cuda()
        hd = torch.from_numpy(h).cuda()
        yd = torch.full_like(xd, 7.0)
        torch.cuda.synchronize()
        stream = side.cuda_stream if on_side else None
        rc = lib.tanb_convolve_no_alloc(xd.data_ptr(), hd.data_ptr(), yd.data_ptr(), C, nb * B, L, B, stream)
        assert rc == cv.AMF_OK, cv.last_error()
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        for c in range(C):
            assert fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) < -120, (call, c)
        ref = _object_path(ctx, x, h, B)
        y[:, :B] *= np.arange(B, dtype=np.float32) / B
        rms = np.sqrt(np.mean(ref.astype(np.float64) ** 2))
        assert np.max(np.abs(y - ref)) <= TOL * rms, (call, np.max(np.abs(y - ref)) / rms)
    # a working set beyond the scratch array is refused with a clear error
    big = torch.zeros(1 << 20, device="cuda")
    rc = lib.tanb_convolve_no_alloc(big.data_ptr(), big.data_ptr(), big.data_ptr(), 64, 4096, 1 << 16, 512, None)
    assert rc == cv.AMF_INVALID_ARG and "scratch" in cv.last_error()
    ctx.Release()
