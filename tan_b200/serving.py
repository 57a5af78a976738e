"""Serving loop over the batched engine, and real-time capacity of both forms.

Sessions (each the equivalent of one TANConvolution: 1-8 channels, IR length
log-uniform in [8192, 524288]) arrive as a Poisson process and live for
exponential lifetimes; each receives IR swaps at a Poisson rate. Every audio
block the loop admits arrivals while the device-memory budget allows (refused
sessions are counted), retires departures, applies pending IR swaps, writes the
block's input, runs one engine block and records the block latency against the
block deadline B / fs. Time is simulated block by block as fast as the device
allows; the latency of a block is the host wall time of everything done for it.

`capacity()` measures the largest number of channels whose p99 block latency
stays under the deadline, for the engine ("batched") and for one
TANConvolution object per session processed in turn ("plain").

    python -m tan_b200.serving --seconds 30 --rate 20 --spectrum fp32
    python -m tan_b200.serving --capacity --ir-length 65536
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import convolution as cv
from . import engine as eng

FS = 48000


class IRPool:
    """Pre-generated exp-decayed Gaussian noise IRs (unit L2 norm per prefix use).
    The running sums of squares are kept, so a prefix's norm costs nothing and
    a request is one scaled copy per channel."""

    def __init__(self, g, n=8, length=524288, rt60=(0.2, 3.0)):
        t = np.arange(length, dtype=np.float64)
        self.irs, self.energy = [], []
        for _ in range(n):
            r = g.uniform(*rt60)
            h = g.standard_normal(length) * np.exp(-np.log(1000.0) * t / (r * FS))
            self.irs.append(h.astype(np.float32))
            self.energy.append(np.cumsum(h * h))

    def get(self, g, C, L):
        out = np.empty((C, L), np.float32)
        for c in range(C):
            i = int(g.integers(len(self.irs)))
            np.multiply(self.irs[i][:L], np.float32(1.0 / np.sqrt(self.energy[i][L - 1])), out=out[c])
        return out


def percentiles(lat_ms):
    a = np.asarray(lat_ms)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
            "p999": float(np.percentile(a, 99.9)), "max": float(a.max())}


def serve(ctx, seconds=30.0, rate=20.0, lifetime=30.0, swap_rate=0.5, block=256, spectrum=eng.SPECTRUM_FP32,
          budget=150 << 30, max_channels=1 << 16, ch_range=(1, 8), len_range=(8192, 524288), seed=20261203 + 4,
          prefill=True, trace=0):
    """Runs the serving loop; returns a dict of latency and occupancy statistics.

    The audio thread admits and retires sessions and runs one engine block per
    block period; a control-plane thread produces IRs and uploads them with
    UpdateResponseTD (asynchronous: a swap lands on the first block after its
    transform finished) and closes retired sessions, as the reference's update
    thread does for TANConvolution. The audio input buffer is filled once (the
    caller's audio I/O would write it in place); the block latency is the host
    wall time of admission + engine block.

    trace=N records the first N sessions admitted in the loop (not prefilled):
    they live to the end, their IR swaps are made on the audio thread with
    BLOCK_UNTIL_READY (so each lands on a known block), and their input rows,
    swap IRs and output rows are returned under "traces", so that a caller can
    check each against the same session run alone."""
    import queue
    import sys
    import threading

    # the audio loop and the control thread share the interpreter: hand it
    # over often, so that the control thread's work delays a block by well
    # under a millisecond rather than by the default 5 ms switch interval
    old_switch = sys.getswitchinterval()
    sys.setswitchinterval(2e-4)
    g = np.random.Generator(np.random.PCG64(seed))
    gw = np.random.Generator(np.random.PCG64(seed + 1))  # the control thread's own stream
    pool = IRPool(g, length=len_range[1])
    e = eng.Engine(ctx, block, spectrum, budget_bytes=budget, max_channels=max_channels)
    e.inp[:] = g.uniform(-1.0, 1.0, e.inp.shape).astype(np.float32)
    deadline_ms = 1000.0 * block / FS
    nblocks = int(seconds * FS / block)
    dt = block / FS
    work = queue.Queue()
    errors = []

    def control():
        while True:
            item = work.get()
            if item is None:
                return
            kind, sess = item
            try:
                if kind == "ir":
                    rc = sess.update_response_td(pool.get(gw, sess.channels, sess.ir_length))
                else:
                    rc = sess.close()
                if rc != cv.AMF_OK:
                    errors.append((kind, rc, cv.last_error()))
            except Exception as ex:  # noqa: BLE001
                errors.append((kind, -1, repr(ex)))
            finally:
                work.task_done()

    ctl = threading.Thread(target=control, daemon=True)
    ctl.start()
    live = {}  # id -> [session, end_time, next_swap_time]
    refused = admitted = 0
    lat, chans = [], []
    t = 0.0
    next_arrival = g.exponential(1.0 / rate)
    traces = {}  # id -> {"session", "x", "events": {block: ir}, "y": [blocks]}
    k_now = 0

    def new_session(now, traced=False):
        nonlocal refused, admitted
        C = int(g.integers(ch_range[0], ch_range[1] + 1))
        L = int(np.exp(g.uniform(np.log(len_range[0]), np.log(len_range[1]))))
        rc, s = e.open_session(C, L)
        if rc != cv.AMF_OK:
            refused += 1
            return
        admitted += 1
        if traced:
            ir = pool.get(g, C, L)
            assert s.update_response_td(ir, block_until_ready=True) == cv.AMF_OK
            traces[s.id] = {"channels": C, "ir_length": L, "x": e.inp[s.slots].copy(), "events": {0: ir},
                            "start": k_now, "y": []}
            live[s.id] = [s, float("inf"), now + g.exponential(1.0 / swap_rate)]
            return
        work.put(("ir", s))
        live[s.id] = [s, now + g.exponential(lifetime), now + g.exponential(1.0 / swap_rate)]

    if prefill:  # start in steady state: rate x lifetime sessions already running
        for _ in range(int(rate * lifetime)):
            new_session(0.0)
        work.join()
        # the prefilled sessions' IRs all take effect on the next block: run
        # it before the loop, which then starts in steady state
        assert e.synchronize() == cv.AMF_OK
        assert e.process() == cv.AMF_OK, cv.last_error()
    for k in range(nblocks):
        k_now = k
        t0 = time.perf_counter()
        while next_arrival <= t:
            new_session(t, traced=len(traces) < trace)
            next_arrival += g.exponential(1.0 / rate)
        for sid in [sid for sid, v in live.items() if v[1] <= t]:
            work.put(("close", live.pop(sid)[0]))
        for sid, v in live.items():
            if v[2] <= t:
                if sid in traces:
                    tr = traces[sid]
                    ir = pool.get(g, tr["channels"], tr["ir_length"])
                    assert v[0].update_response_td(ir, block_until_ready=True) == cv.AMF_OK
                    tr["events"][k - tr["start"]] = ir
                else:
                    work.put(("ir", v[0]))
                v[2] = t + g.exponential(1.0 / swap_rate)
        if live:  # an idle engine has no block to run
            rc = e.process()
            assert rc == cv.AMF_OK, cv.last_error()
        lat.append(1000.0 * (time.perf_counter() - t0))
        for sid, tr in traces.items():
            tr["y"].append(e.out[live[sid][0].slots].copy())
        chans.append(e.info()["channels"])
        t += dt
    work.put(None)
    ctl.join()
    times = e.block_times()
    sys.setswitchinterval(old_switch)
    e.synchronize()
    info = e.info()
    e.release()
    lat = np.asarray(lat)
    out = {"blocks": nblocks, "deadline_ms": deadline_ms, "latency_ms": percentiles(lat),
           "deadline_misses": int((lat > deadline_ms).sum()), "concurrent_channels_mean": float(np.mean(chans)),
           "concurrent_channels_max": int(np.max(chans)), "admitted": admitted, "refused": refused,
           "control_errors": errors[:5], "arena_bytes_end": info["arena_bytes"],
           "block_graphs_built": int(times["graph_builds"]),
           "spectrum": ["fp32", "fp16", "bf16", "fp24"][spectrum]}
    if trace:
        out["traces"] = [dict(tr, y=np.concatenate(tr["y"], axis=1)) for tr in traces.values()]
    return out


class EngineSlots:
    """A rank's engine as the sharding control plane sees it: open(spec) ->
    session or None (refused by the budget or the slot table), close(session),
    snapshot(session) -> bytes or None (the session's state; uniformly
    partitioned sessions) and restore(spec, bytes) -> session or None."""

    def __init__(self, engine):
        self.engine = engine

    def open(self, spec):
        if spec.levels:
            rc, sess = self.engine.open_session_nu(spec.channels, spec.ir_length, list(spec.levels))
        else:
            rc, sess = self.engine.open_session(spec.channels, spec.ir_length)
        return sess if rc == cv.AMF_OK else None

    def close(self, sess):
        sess.close()

    def snapshot(self, sess):
        rc, buf = sess.snapshot()
        return buf.tobytes() if rc == cv.AMF_OK else None

    def restore(self, spec, blob):
        rc, sess = self.engine.open_session_restore(np.frombuffer(blob, np.uint8))
        return sess if rc == cv.AMF_OK else None


def serve_sharded(pg, ctx, sessions=600, blocks=1500, swap_rate=0.5, block=256, spectrum=eng.SPECTRUM_FP32,
                  budget=150 << 30, ch_range=(1, 8), len_range=(8192, 524288), seed=20261203 + 4):
    """Sessions sharded over the ranks of `pg` (one GPU each): rank 0 draws the
    session mix (channels, IR lengths), sharding.RankServer places it by the
    engines' admission rule (refused sessions re-placed on the other ranks),
    and every rank serves its shard with its own engine for `blocks` blocks,
    with Poisson IR swaps. No audio crosses GPUs; the per-rank block latencies
    are gathered to rank 0. Returns (on every rank) the latency percentiles
    over all ranks' blocks, and the channels per rank."""
    import torch

    from . import sharding as sh

    rank, world = pg.get_rank(), pg.get_world_size()
    g = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for sid in range(sessions):
        C = int(g.integers(ch_range[0], ch_range[1] + 1))
        L = int(np.exp(g.uniform(np.log(len_range[0]), np.log(len_range[1]))))
        specs.append(sh.SessionSpec(sid, C, L))
    e = eng.Engine(ctx, block, spectrum, budget_bytes=budget, max_channels=1 << 16)
    srv = sh.RankServer(pg, EngineSlots(e), block, budget)
    placement = srv.place(specs)
    gl = np.random.Generator(np.random.PCG64(seed + 100 + rank))
    pool = IRPool(gl, length=len_range[1])
    mine = {sid: s for sid, s in srv.handles.items()}
    for sid, sess in mine.items():
        sess.update_response_td(pool.get(gl, sess.channels, sess.ir_length), block_until_ready=True)
    e.inp[:] = gl.uniform(-1.0, 1.0, e.inp.shape).astype(np.float32)
    dt = block / FS
    next_swap = {sid: gl.exponential(1.0 / swap_rate) for sid in mine}
    lat = []
    t = 0.0
    for k in range(blocks):
        t0 = time.perf_counter()
        for sid, sess in mine.items():
            if next_swap[sid] <= t:
                sess.update_response_td(pool.get(gl, sess.channels, sess.ir_length))
                next_swap[sid] = t + gl.exponential(1.0 / swap_rate)
        if mine:
            assert e.process() == cv.AMF_OK, cv.last_error()
        lat.append(1000.0 * (time.perf_counter() - t0))
        t += dt
    chans = e.info()["channels"]
    e.release()
    all_lat = [None] * world
    pg.all_gather_object(all_lat, (lat, chans))
    lats = np.concatenate([np.asarray(a) for a, _ in all_lat])
    torch.cuda.synchronize()
    return {"ranks": world, "blocks": blocks, "deadline_ms": 1000.0 * block / FS, "latency_ms": percentiles(lats),
            "deadline_misses": int((lats > 1000.0 * block / FS).sum()),
            "channels_per_rank": [c for _, c in all_lat], "sessions": sessions,
            "unplaced": int(sum(1 for r in placement.values() if r < 0))}


def _block_latencies_batched(ctx, nsess, C, L, block, spectrum, blocks, g, pool):
    e = eng.Engine(ctx, block, spectrum, budget_bytes=170 << 30, max_channels=nsess * C + 8)
    sess = []
    for _ in range(nsess):
        rc, s = e.open_session(C, L)
        if rc != cv.AMF_OK:
            e.release()
            return None
        s.update_response_td(pool.get(g, C, L), block_until_ready=True)
        sess.append(s)
    x = g.uniform(-1, 1, (nsess * C, block)).astype(np.float32)
    lat = []
    for k in range(blocks + 5):
        t0 = time.perf_counter()
        assert e.write_input(0, x) == cv.AMF_OK  # the block's input, every channel
        assert e.process() == cv.AMF_OK
        if k >= 5:
            lat.append(1000.0 * (time.perf_counter() - t0))
    e.release()
    return np.asarray(lat)


def _block_latencies_plain(ctx, nsess, C, L, block, blocks, g, pool):
    from . import autotune

    convs = []
    for _ in range(nsess):
        try:  # the drop-in with its autotuned tail tiling for this shape
            conv = autotune.tuned(ctx, cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, block, C)
        except cv.TANError:
            for c in convs:
                c.Release()
            return None
        conv.UpdateResponseTD(pool.get(g, C, L), L)
        convs.append(conv)
    x = g.uniform(-1, 1, (C, block)).astype(np.float32)
    y = np.zeros_like(x)
    import ctypes

    lib = cv.lib()
    rin = (ctypes.c_void_p * C)(*[x[c].ctypes.data for c in range(C)])
    rout = (ctypes.c_void_p * C)(*[y[c].ctypes.data for c in range(C)])
    done = ctypes.c_size_t(0)
    lat = []
    for k in range(blocks + 5):
        t0 = time.perf_counter()
        for conv in convs:
            rc = lib.tanb_convolution_process(conv._h, rin, rout, block, None, ctypes.byref(done))
            assert rc == cv.AMF_OK
        if k >= 5:
            lat.append(1000.0 * (time.perf_counter() - t0))
    for c in convs:
        c.Release()
    return np.asarray(lat)


def _block_latencies_plain_one(ctx, nsess, C, L, block, blocks, g, pool):
    """One drop-in object holding every channel (nsess * C), host rows."""
    from . import autotune

    n = nsess * C
    try:
        conv = autotune.tuned(ctx, cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, block, n)
    except cv.TANError:
        return None
    import ctypes

    lib = cv.lib()
    # one IR row for every channel (the transform and the streamed bytes are
    # the same as with distinct rows; the host keeps one row instead of n)
    h = pool.get(g, 1, L)
    rows = (ctypes.c_void_p * n)(*([h[0].ctypes.data] * n))
    assert lib.tanb_convolution_update_response_td(conv._h, rows, L, None, 0) == cv.AMF_OK
    x = g.uniform(-1, 1, (n, block)).astype(np.float32)
    y = np.zeros_like(x)
    rin = (ctypes.c_void_p * n)(*[x[c].ctypes.data for c in range(n)])
    rout = (ctypes.c_void_p * n)(*[y[c].ctypes.data for c in range(n)])
    done = ctypes.c_size_t(0)
    lat = []
    for k in range(blocks + 5):
        t0 = time.perf_counter()
        rc = lib.tanb_convolution_process(conv._h, rin, rout, block, None, ctypes.byref(done))
        assert rc == cv.AMF_OK
        if k >= 5:
            lat.append(1000.0 * (time.perf_counter() - t0))
    conv.Release()
    return np.asarray(lat)


def capacity(ctx, form="batched", C=4, L=65536, block=256, spectrum=eng.SPECTRUM_FP32, blocks=200,
             seed=20261203 + 5, start=4):
    """Largest channel count (sessions of C channels, IR length L) whose p99 block
    latency is under the deadline; doubling then bisection on the session count.
    form: "batched" (the engine), "plain" (one TANConvolution per session,
    processed in turn) or "plain_one" (one TANConvolution holding every
    channel)."""
    g = np.random.Generator(np.random.PCG64(seed))
    pool = IRPool(g, n=4, length=L)
    deadline = 1000.0 * block / FS

    def ok(n):
        if form == "batched":
            lat = _block_latencies_batched(ctx, n, C, L, block, spectrum, blocks, g, pool)
        elif form == "plain_one":
            lat = _block_latencies_plain_one(ctx, n, C, L, block, blocks, g, pool)
        else:
            lat = _block_latencies_plain(ctx, n, C, L, block, blocks, g, pool)
        if lat is None:
            return False, None
        p99 = float(np.percentile(lat, 99))
        return p99 < deadline, p99

    lo, hi = 0, start
    last = {}
    while True:
        good, p99 = ok(hi)
        last[hi] = p99
        if not good:
            break
        lo, hi = hi, hi * 2
        if hi * C > (1 << 17):
            break
    while hi - lo > max(1, lo // 32):
        mid = (lo + hi) // 2
        good, p99 = ok(mid)
        last[mid] = p99
        lo, hi = (mid, hi) if good else (lo, mid)
    return {"form": form, "max_realtime_channels": lo * C, "sessions": lo, "channels_per_session": C,
            "ir_length": L, "block": block, "deadline_ms": deadline, "p99_at": {str(k): v for k, v in last.items()}}


def mac_roofline(ctx, channels, C=4, L=48000, block=256, spectrum=eng.SPECTRUM_FP32, blocks=48,
                 seed=20261203 + 5):
    """Device time of the engine's block launch with `channels` resident
    channels (sessions of C channels, IR length L): CUDA events around each
    block on the engine's stream, inputs and outputs in device memory. The
    working set (IR spectra and delay lines of every channel) is far larger
    than L2, so every block streams it from HBM. Returns the algorithmic bytes
    of one launch (IR spectra, delay line, partial rows, I/O) and the mean
    launch time."""
    import torch

    g = np.random.Generator(np.random.PCG64(seed))
    pool = IRPool(g, n=4, length=L)
    nsess = max(1, channels // C)
    e = eng.Engine(ctx, block, spectrum, budget_bytes=170 << 30, max_channels=nsess * C + 8)
    try:
        for i in range(nsess):
            rc, s = e.open_session(C, L)
            if rc != cv.AMF_OK:
                raise RuntimeError("open_session failed after %d sessions" % i)
            s.update_response_td(pool.get(g, C, L), block_until_ready=True)
        n = nsess * C
        d_in = torch.empty((n, block), dtype=torch.float32, device="cuda").uniform_(-1, 1)
        d_out = torch.empty_like(d_in)
        for _ in range(5):
            assert e.process_device(d_in.data_ptr(), d_out.data_ptr()) == cv.AMF_OK
        e.synchronize()
        e.profile(True)
        e.profile_read()
        for _ in range(blocks):
            assert e.process_device(d_in.data_ptr(), d_out.data_ptr()) == cv.AMF_OK
        p = e.profile_read()
        e.profile(False)
        info = e.info()
    finally:
        e.release()
    us = 1000.0 * p["block_ms"] / max(1, p["timed"])
    return {"channels": n, "ir_length": L, "block": block, "bytes_per_launch": int(info["block_bytes"]),
            "avg_launch_us": us, "launches_timed": int(p["timed"]),
            "achieved_gbs": info["block_bytes"] / (us * 1e-6) / 1e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seconds", type=float, default=30.0)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--spectrum", choices=["fp32", "fp16", "bf16", "fp24"], default="fp32")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--capacity", action="store_true")
    ap.add_argument("--form", choices=["batched", "plain", "plain_one"], default="batched")
    ap.add_argument("--ir-length", type=int, default=65536)
    ap.add_argument("--channels", type=int, default=4)
    ap.add_argument("--mac-roofline", type=int, default=0, metavar="CHANNELS",
                    help="time the engine's block launch with this many resident channels")
    a = ap.parse_args()
    spec = {"fp32": eng.SPECTRUM_FP32, "fp16": eng.SPECTRUM_FP16, "bf16": eng.SPECTRUM_BF16,
            "fp24": eng.SPECTRUM_FP24}[a.spectrum]
    ctx = cv.TANContext(0)
    if a.mac_roofline:
        r = mac_roofline(ctx, a.mac_roofline, a.channels, a.ir_length, spectrum=spec)
    elif a.capacity:
        r = capacity(ctx, a.form, a.channels, a.ir_length, spectrum=spec)
    else:
        r = serve(ctx, a.seconds, a.rate, spectrum=spec, budget=int(a.budget_gb * (1 << 30)))
    print(json.dumps(r))


if __name__ == "__main__":
    main()
