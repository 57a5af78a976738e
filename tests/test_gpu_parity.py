"""GPU parity: the CUDA path through the C ABI against the oracle (the C++
restatement of TAN's CPU uniformly-partitioned path, and the FP64 statement).

Tolerances: max |gpu - restatement| <= 1e-5 x rms(restatement output) on every
block (steady state and swap blocks alike, both implement the same crossfade);
error vs FP64 <= -120 dB for FP32 spectra; delta-IR known answers within 2e-6.
"""
import numpy as np
import pytest

from oracle import fp64, ref
from tan_b200 import convolution as cv
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-5


def make(ctx, L, B, C, method=cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM):
    conv = cv.TANConvolution(ctx)
    rc = conv.Init(method, L, B, C)
    assert rc == cv.AMF_OK, (rc, cv.last_error())
    return conv


def test_known_answer_delta_irs(tan_ctx):
    h = H.delta_irs()
    taps = H.golden_taps()["channels"]
    x = H.pulsetrain(2)
    B = 128
    conv = make(tan_ctx, h.shape[1], B, 2)
    y, codes = H.run_stream(conv, x, B, events={0: (h, None)}, per_call_blocks=8)
    assert all(c == 0 for c in codes)
    T = y.shape[1]
    for c in range(2):
        exp = np.zeros(T, np.float64)
        for t in taps[c]:
            exp[t["index"]:] += t["value"] * x[c, : T - t["index"]].astype(np.float64)
        exp[:B] *= np.arange(B) / B
        assert np.max(np.abs(y[c] - exp)) < 2e-6
    conv.Release()


def test_two_channels_b1024_ir8192_parity_with_restatement(tan_ctx):
    """2 channels, B=1024, IR 8192 (8 partitions), 200 blocks, RT60 0.3 s."""
    g = H.rng(20261203 + 0)
    C, B, L, nb = 2, 1024, 8192, 200
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L, (0.3, 0.3))
    gpu = make(tan_ctx, L, B, C)
    y, codes = H.run_stream(gpu, x, B, {0: (h, None)})
    assert all(c == 0 for c in codes)
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, {0: (h, None)})
    assert H.rel_err(y, yr) < TOL
    exp = fp64.stream_fp64(x, B, [(0, {c: h[c] for c in range(C)})])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120
    gpu.Release()


def test_time_varying_swaps_parity(tan_ctx):
    """The 64-channel bench shape reduced in channels/blocks: B=512, IR 65536 (128 partitions),
    IR replaced every 32 blocks with a one-block crossfade."""
    g = H.rng(20261203 + 1)
    C, B, L, nb = 4, 512, 65536, 100
    x = H.noise(g, C, nb * B)
    events, fp_events = {}, []
    for k in range(0, nb, 32):
        h = H.irs(g, C, L, (0.2, 1.5))
        events[k] = (h, None)
        fp_events.append((k, {c: h[c] for c in range(C)}))
    gpu = make(tan_ctx, L, B, C)
    y, codes = H.run_stream(gpu, x, B, events, per_call_blocks=5)
    assert all(c == 0 for c in codes)
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, events)
    assert H.rel_err(y, yr) < TOL
    exp = fp64.stream_fp64(x, B, fp_events)
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120
    gpu.Release()


@pytest.mark.parametrize("B", [32, 64, 256, 512, 2048, 4096, 8192])
@pytest.mark.parametrize("Lfac", [0.5, 1.0, 2.0, 3.3])  # 2.0: two partitions, no tail launch
def test_sizes_sweep(tan_ctx, B, Lfac):
    L = max(1, int(B * Lfac))
    C = 3
    g = H.rng(B * 10 + int(Lfac * 10))
    nb = 9
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    events = {0: (h0, None), 4: (h1, None)}
    gpu = make(tan_ctx, L, B, C)
    y, codes = H.run_stream(gpu, x, B, events, per_call_blocks=3)
    assert all(c == 0 for c in codes)
    exp = fp64.stream_fp64(x, B, [(0, {c: h0[c] for c in range(C)}), (4, {c: h1[c] for c in range(C)})])
    for c in range(C):
        assert fp64.error_db(y[c], exp[c]) < -120, (c, fp64.error_db(y[c], exp[c]))
    gpu.Release()


def test_flags_match_restatement(tan_ctx):
    """STOP_INPUT ring-out, FLUSH_STREAM, partial IR updates, free channels."""
    g = H.rng(99)
    C, B, L, nb = 4, 256, 1500, 30
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    events = {0: (h0, None), 7: (h1, np.array([0, 1, 0, 3], np.uint32))}
    flags = []
    for k in range(nb):
        f = np.zeros(C, np.uint32)
        if 3 <= k < 20:
            f[1] = 1  # stop channel 1 -> rings out for nextpow2(L) = 2048 samples = 8 blocks
        if k == 10:
            f[2] = 2  # flush channel 2
        if k >= 12:
            f[3] = 1 | 2  # stop + flush channel 3: free at once
        flags.append(f)
    gpu = make(tan_ctx, L, B, C)
    oracle = ref.RefConvolution(L, B, C)
    sentinel = 3.25
    outs = []
    for conv in (gpu, oracle):
        y = np.full((C, nb * B), sentinel, np.float32)
        for k in range(nb):
            if k == 19:  # channel 1 rang out (blocks 3..10) and channel 3 is free: first free is 1
                free = conv.GetNextFreeChannel(flags[k]) if conv is gpu else conv.next_free_channel(flags[k])
                assert free == (0, 1)
            if k in events:
                ir, fl = events[k]
                rc = conv.UpdateResponseTD(ir, L, fl) if conv is gpu else conv.update_response_td(ir, fl)
                assert rc == 0
            xs = np.ascontiguousarray(x[:, k * B:(k + 1) * B])
            ys = np.ascontiguousarray(y[:, k * B:(k + 1) * B])
            if conv is gpu:
                rc, done = conv.Process(xs, ys, B, flags[k])
            else:
                rc, ys, done = conv.process(xs, flags[k], ys)
            assert rc == 0 and done == B
            y[:, k * B:(k + 1) * B] = ys
        outs.append(y)
        free = conv.GetNextFreeChannel(flags[-1]) if conv is gpu else conv.next_free_channel(flags[-1])
        assert free == (0, 3)
    y, yr = outs
    assert np.array_equal(y == sentinel, yr == sentinel)
    live = yr != sentinel
    assert np.max(np.abs(y[live] - yr[live])) < TOL * np.sqrt(np.mean(yr[live].astype(np.float64) ** 2))
    gpu.Release()


def test_all_channels_stopped_is_wrong_state(tan_ctx):
    gpu = make(tan_ctx, 512, 128, 2)
    x = np.zeros((2, 128), np.float32)
    y = np.zeros_like(x)
    rc, done = gpu.Process(x, y, 128, np.array([3, 3], np.uint32))
    assert rc == cv.AMF_WRONG_STATE and done == 0
    gpu.Release()


def test_error_codes(tan_ctx):
    conv = cv.TANConvolution(tan_ctx)
    x = np.zeros((2, 256), np.float32)
    conv.channels = 2
    assert conv.UpdateResponseTD(x, 256) == cv.AMF_NOT_INITIALIZED
    assert conv.Init(1, 1024, 0, 2) == cv.AMF_INVALID_ARG
    assert conv.Init(1, 1024, 100, 2) == cv.AMF_INVALID_ARG  # not a power of two
    assert conv.Init(1, 0, 256, 2) == cv.AMF_INVALID_ARG
    assert conv.Init(42, 1024, 256, 2) == cv.AMF_NOT_SUPPORTED
    assert conv.Init(1, 1024, 256, 2) == cv.AMF_OK
    assert conv.Init(1, 1024, 256, 2) == cv.AMF_ALREADY_INITIALIZED
    assert conv.UpdateResponseTD(np.zeros((2, 2048), np.float32), 2048) == cv.AMF_INVALID_ARG  # longer than Init
    assert conv.UpdateResponseFD(x, 256) == cv.AMF_NOT_SUPPORTED
    rc, done = conv.ProcessDirect(x, x, x.copy(), 256)
    assert rc == cv.AMF_NOT_SUPPORTED
    y = np.zeros_like(x)
    rc, done = conv.Process(x[:, :100].copy(), y[:, :100].copy(), 100)
    assert rc == cv.AMF_OK and done == 0
    assert conv.Terminate() == cv.AMF_OK
    assert conv.Init(1, 1024, 256, 2) == cv.AMF_WRONG_STATE
    conv.Release()


def test_finalize_mode_and_device_buffers_match_host_path(tan_ctx):
    import torch

    g = H.rng(5)
    C, B, L, nb = 3, 256, 3000, 12
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    base = make(tan_ctx, L, B, C)
    y0, _ = H.run_stream(base, x, B, {0: (h, None)})
    fin = make(tan_ctx, L, B, C, cv.TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM | cv.TAN_CONVOLUTION_METHOD_USE_PROCESS_FINALIZE)
    assert fin.UpdateResponseTD(h, L) == 0
    y1 = np.zeros_like(y0)
    for k in range(nb):
        xs = np.ascontiguousarray(x[:, k * B:(k + 1) * B])
        ys = np.zeros_like(xs)
        rc, done = fin.Process(xs, ys, B)
        assert rc == 0 and done == B
        assert fin.ProcessFinalize() == 0
        y1[:, k * B:(k + 1) * B] = ys
    assert np.array_equal(y0, y1)
    dev = make(tan_ctx, L, B, C, cv.TAN_CONVOLUTION_METHOD_FHT_UNIFORM_HEAD_TAIL)
    hd = torch.from_numpy(h).cuda()
    assert dev.UpdateResponseTDDevice(hd, L) == 0
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    rc, done = dev.ProcessDevice(xd, yd, nb * B)
    assert rc == 0 and done == nb * B
    assert dev.Synchronize() == 0
    assert np.array_equal(yd.cpu().numpy(), y0)
    # host in, device out
    hyb = make(tan_ctx, L, B, C)
    assert hyb.UpdateResponseTD(h, L) == 0
    yd2 = torch.zeros_like(xd)
    rc, done = hyb.ProcessHostToDevice(x, yd2, nb * B)
    assert rc == 0 and done == nb * B
    assert np.array_equal(yd2.cpu().numpy(), y0)
    for c_ in (base, fin, dev, hyb):
        c_.Release()


@pytest.mark.parametrize("C", [128, 160])
def test_channel_counts_around_the_parameter_descriptor_limit(tan_ctx, C):
    """Up to 128 channels the per-block channel states travel as kernel
    parameters; beyond that as device tables. Both match the restatement with
    channel flags and an IR swap, and the host, host-to-device and device
    overloads give the same samples (multi-block calls included)."""
    import torch

    g = H.rng(700 + C)
    B, L, nb = 256, 3000, 12
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    events = {0: (h0, None), 5: (h1, None)}
    flags = []
    for k in range(nb):
        f = np.zeros(C, np.uint32)
        if 2 <= k < 9:
            f[7] = 1  # STOP_INPUT: rings out
        if k == 6:
            f[C - 1] = 2  # FLUSH_STREAM
        flags.append(f)
    gpu = make(tan_ctx, L, B, C)
    y, codes = H.run_stream(gpu, x, B, events, flags_per_block=flags)
    assert all(c == 0 for c in codes)
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, events, flags_per_block=flags)
    assert H.rel_err(y, yr) < TOL
    # no flags: host rows in 4-block calls vs device and host-to-device overloads
    host = make(tan_ctx, L, B, C)
    y0, codes = H.run_stream(host, x, B, events, per_call_blocks=4)
    assert all(c == 0 for c in codes)
    dev = make(tan_ctx, L, B, C)
    hyb = make(tan_ctx, L, B, C)
    xd = torch.from_numpy(x).cuda()
    yd, yh = torch.zeros_like(xd), torch.zeros_like(xd)
    for k0, k1 in ((0, 5), (5, nb)):
        h = events[k0][0]
        assert dev.UpdateResponseTDDevice(torch.from_numpy(h).cuda(), L) == 0
        assert hyb.UpdateResponseTD(h, L) == 0
        rc, done = dev.ProcessDevice([xd[c, k0 * B:k1 * B] for c in range(C)],
                                     [yd[c, k0 * B:k1 * B] for c in range(C)], (k1 - k0) * B)
        assert rc == 0 and done == (k1 - k0) * B
        rc, done = hyb.ProcessHostToDevice(np.ascontiguousarray(x[:, k0 * B:k1 * B]),
                                           [yh[c, k0 * B:k1 * B] for c in range(C)], (k1 - k0) * B)
        assert rc == 0 and done == (k1 - k0) * B
    assert dev.Synchronize() == 0 and hyb.Synchronize() == 0
    assert np.array_equal(yd.cpu().numpy(), y0)
    assert np.array_equal(yh.cpu().numpy(), y0)
    for c_ in (gpu, host, dev, hyb):
        c_.Release()


def test_mixed_io_overloads_on_one_object_equal_host_only(tan_ctx):
    """Host-row calls return once their heads have signalled, while the tail
    behind them still runs; host-to-device and device calls in between reuse
    the same staging rows. Alternating the overloads (single and multi-block
    calls, an IR swap in the middle) gives the host-only samples exactly."""
    import torch

    g = H.rng(31)
    C, B, L, nb = 5, 256, 6000, 24
    x = H.noise(g, C, nb * B)
    h0, h1 = H.irs(g, C, L), H.irs(g, C, L)
    ref_conv = make(tan_ctx, L, B, C)
    y0, codes = H.run_stream(ref_conv, x, B, {0: (h0, None), 11: (h1, None)}, per_call_blocks=1)
    assert all(c == 0 for c in codes)
    mix = make(tan_ctx, L, B, C)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    y = np.zeros_like(y0)
    plan = [(0, 1, "host"), (1, 3, "h2d"), (3, 6, "host"), (6, 7, "dev"), (7, 9, "host"), (9, 11, "h2d"),
            (11, 12, "host"), (12, 15, "dev"), (15, 16, "h2d"), (16, 20, "host"), (20, 24, "dev")]
    for k0, k1, kind in plan:
        if k0 == 0:
            assert mix.UpdateResponseTD(h0, L) == 0
        if k0 == 11:
            assert mix.UpdateResponseTD(h1, L) == 0
        n = (k1 - k0) * B
        xs = np.ascontiguousarray(x[:, k0 * B:k1 * B])
        if kind == "host":
            ys = np.zeros_like(xs)
            rc, done = mix.Process(xs, ys, n)
            y[:, k0 * B:k1 * B] = ys
        elif kind == "h2d":
            rc, done = mix.ProcessHostToDevice(xs, [yd[c, k0 * B:k1 * B] for c in range(C)], n)
        else:
            rc, done = mix.ProcessDevice([xd[c, k0 * B:k1 * B] for c in range(C)],
                                         [yd[c, k0 * B:k1 * B] for c in range(C)], n)
        assert rc == 0 and done == n
    assert mix.Synchronize() == 0
    yd_h = yd.cpu().numpy()
    for k0, k1, kind in plan:
        if kind != "host":
            y[:, k0 * B:k1 * B] = yd_h[:, k0 * B:k1 * B]
    assert np.array_equal(y, y0)
    ref_conv.Release()
    mix.Release()


def test_multi_block_calls_equal_single_block_calls(tan_ctx):
    g = H.rng(8)
    C, B, L, nb = 2, 128, 4096, 40
    x = H.noise(g, C, nb * B)
    h = H.irs(g, C, L)
    a = make(tan_ctx, L, B, C)
    ya, _ = H.run_stream(a, x, B, {0: (h, None)}, per_call_blocks=1)
    b = make(tan_ctx, L, B, C)
    assert b.UpdateResponseTD(h, L) == 0
    yb = np.zeros_like(ya)
    rc, done = b.Process(x, yb, nb * B + 77)
    assert rc == 0 and done == nb * B
    assert np.array_equal(ya, yb)
    a.Release()
    b.Release()


def test_full_size_64ch_b512_ir65536_properties(tan_ctx):
    """64 channels, B=512, IR 65536: linearity and the delta-IR known answer at
    full size (size-independent properties; the oracle covers smaller sizes)."""
    g = H.rng(20261203 + 1)
    C, B, L, nb = 64, 512, 65536, 96
    x1, x2 = H.noise(g, C, nb * B), H.noise(g, C, nb * B)
    h = H.irs(g, C, L, (0.2, 1.5))
    outs = []
    for x in (x1, x2, (0.5 * x1 - 2.0 * x2).astype(np.float32)):
        conv = make(tan_ctx, L, B, C)
        y, codes = H.run_stream(conv, x, B, {0: (h, None)}, per_call_blocks=8)
        assert all(c == 0 for c in codes)
        outs.append(y.astype(np.float64))
        conv.Release()
    lin = 0.5 * outs[0] - 2.0 * outs[1]
    assert np.max(np.abs(outs[2] - lin)) < 1e-5 * np.sqrt(np.mean(lin ** 2))
    # exact check of a few channels against FP64
    exp = fp64.stream_fp64(x1[:4], B, [(0, {c: h[c] for c in range(4)})])
    for c in range(4):
        assert fp64.error_db(outs[0][c], exp[c]) < -120
    # delta IR at full length: pure delay of 40000 samples
    d = np.zeros((C, L), np.float32)
    d[:, 40000] = 1.0
    conv = make(tan_ctx, L, B, C)
    y, _ = H.run_stream(conv, x1, B, {0: (d, None)}, per_call_blocks=8)
    T = x1.shape[1]
    assert T > 40000
    assert np.max(np.abs(y[:, 40000:] - x1[:, : T - 40000])) < 1e-6
    conv.Release()


@pytest.mark.parametrize("B,L", [(256, 5000), (512, 20000), (1024, 9000)])
def test_every_tail_tiling_matches_restatement(tan_ctx, B, L):
    """Every compiled tail tiling (register-load and cp.async.bulk pipelines)
    gives the restatement's output within tolerance, swaps included."""
    g = H.rng(B + L)
    C, nb = 3, 10
    x = H.noise(g, C, nb * B)
    events = {0: (H.irs(g, C, L), None), 6: (H.irs(g, C, L), None)}
    oracle = ref.RefConvolution(L, B, C, threads=4)
    yr, _ = H.run_stream(oracle, x, B, events)
    idx = 0
    tested = 0
    while True:
        conv = make(tan_ctx, L, B, C)
        rc, tiling = conv.tiling(idx)
        if rc != cv.AMF_OK:
            conv.Release()
            break
        if tiling[0] <= B // 2:
            y, codes = H.run_stream(conv, x, B, events, per_call_blocks=3)
            assert all(c == 0 for c in codes), (tiling, cv.last_error())
            assert conv.Synchronize() == 0
            assert H.rel_err(y, yr) < TOL, tiling
            tested += 1
        conv.Release()
        idx += 1
    assert tested >= 10


@pytest.mark.parametrize("n_ir", [1, 777, 2999, 3000])
def test_device_rows_update_equals_host_rows_update(tan_ctx, n_ir):
    """UpdateResponseTD from device rows (read in place at any 4-byte offset,
    zero past n) gives bit-identical outputs to the host-row update, for odd
    and short lengths, with a swap mid-stream that skips a stopped channel."""
    import torch

    g = H.rng(60 + n_ir)
    C, B, L, nb = 3, 256, 3000, 14
    x = H.noise(g, C, nb * B)
    h0 = np.ascontiguousarray(H.irs(g, C, L)[:, :n_ir])
    h1 = np.ascontiguousarray(H.irs(g, C, L)[:, :n_ir])
    stop1 = np.array([0, cv.TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT, 0], np.uint32)
    host = make(tan_ctx, L, B, C)
    y_host, _ = H.run_stream(host, x, B, {0: (h0, None), 7: (h1, stop1)})
    dev = make(tan_ctx, L, B, C)
    # rows one float past the start of a wider buffer: no alignment beyond 4 bytes
    wide = torch.zeros((2, C, n_ir + 3), dtype=torch.float32, device="cuda")
    wide[0, :, 1:n_ir + 1] = torch.from_numpy(h0)
    wide[1, :, 1:n_ir + 1] = torch.from_numpy(h1)
    rows = [[wide[s, c].data_ptr() + 4 for c in range(C)] for s in range(2)]
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    for k in range(nb):
        if k == 0:
            assert dev.UpdateResponseTDDevice(rows[0], n_ir) == 0
        if k == 7:
            assert dev.UpdateResponseTDDevice(rows[1], n_ir, stop1) == 0
        rc, done = dev.ProcessDevice([xd[c, k * B:(k + 1) * B] for c in range(C)],
                                     [yd[c, k * B:(k + 1) * B] for c in range(C)], B)
        assert rc == 0 and done == B
    assert dev.Synchronize() == 0
    assert np.array_equal(yd.cpu().numpy(), y_host)
    host.Release()
    dev.Release()
