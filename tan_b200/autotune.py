"""Autotuner for the partition multiply-accumulate (the tail kernel).

For one shape (block B, IR length L, channels C) it runs the convolution on the
device with every compiled tail tiling, timing whole blocks (head plus the tail
that overlaps it) with CUDA events on the object's stream, L2 flushed before
every timed block, and keeps the tiling with the shortest block time. Results are cached in tuning.json next to this file, keyed by shape;
TANConvolution objects created through `tuned()` apply the cached choice.

    python -m tan_b200.autotune --block 512 --length 65536 --channels 64
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import convolution as cv
from . import nupols
from .convolution import AMF_OK

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")


def key(B: int, L: int, C: int) -> str:
    P = max(1, -(-L // B))
    return f"B{B}_P{P}_C{C}"


def load_cache() -> dict:
    if os.path.exists(CACHE):
        with open(CACHE) as f:
            return json.load(f)
    return {}


def save_cache(d: dict) -> None:
    with open(CACHE, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


def measure(ctx, B: int, L: int, C: int, steps: int = 120, warmup: int = 8, seed: int = 7):
    """Returns [(index, (ux, sy, depth), mean block us, mean tail us)] for every
    compiled tiling. The block time is one Process call on device buffers (the
    head, then the tail launched behind it so that the two overlap), timed with
    CUDA events around the call; the tail time comes from a second pass with
    events around each kernel launch (the tail then runs after its head)."""
    import torch

    g = np.random.Generator(np.random.PCG64(seed))
    dev = ctx.device
    h = torch.from_numpy((g.standard_normal((C, L)) * 0.01).astype(np.float32)).to(f"cuda:{dev}")
    x = torch.from_numpy(g.uniform(-1, 1, (C, B)).astype(np.float32)).to(f"cuda:{dev}")
    y = torch.zeros_like(x)
    flush_w = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{dev}")
    flush_r = torch.ones(64 << 20, dtype=torch.float32, device=f"cuda:{dev}")
    flush_r2 = torch.ones(64 << 20, dtype=torch.float32, device=f"cuda:{dev}")
    results = []
    idx = 0
    while True:
        conv = cv.TANConvolution(ctx)
        assert conv.Init(cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C) == cv.AMF_OK, cv.last_error()
        rc, tiling = conv.tiling(idx)
        if rc != cv.AMF_OK:
            conv.Release()
            break
        if tiling[0] > B // 2:  # more units per CTA row than the block has bin pairs
            conv.Release()
            idx += 1
            continue
        assert conv.UpdateResponseTDDevice(h, L) == 0
        stream = torch.cuda.ExternalStream(conv.stream(), device=dev)

        def flush():
            # a 256 MiB write, then two 256 MiB reads, so that no dirty line of
            # the write is left in L2 to be written back inside a timed block
            with torch.cuda.stream(stream):
                flush_w.zero_()
                flush_r.sum()
                flush_r2.sum()

        for _ in range(warmup):
            flush()
            assert conv.ProcessDevice(x, y, B)[0] == 0
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in ev:
            flush()
            a.record(stream)
            assert conv.ProcessDevice(x, y, B)[0] == 0
            b.record(stream)
        conv.Synchronize()
        torch.cuda.synchronize()
        block_us = 1000.0 * sum(a.elapsed_time(b) for a, b in ev) / steps
        conv.profile_read()
        conv.profile(True)
        for _ in range(steps):
            flush()
            assert conv.ProcessDevice(x, y, B)[0] == 0
        conv.Synchronize()
        conv.profile(False)
        p = conv.profile_read()["tail"]
        results.append((idx, tiling, block_us, 1000.0 * p["ms"] / max(1, p["timed"])))
        conv.Release()
        idx += 1
    return results


def tune(ctx, B: int, L: int, C: int, write: bool = True) -> dict:
    """Chooses the tiling with the shortest block time (head + overlapped tail)."""
    res = measure(ctx, B, L, C)
    best = min(res, key=lambda r: r[2])
    P = max(1, -(-L // B))
    bytes_per_launch = C * (max(0, P - 2) * B * 16 + B * 8)  # the tail streams partitions 2..P-1
    entry = {"index": best[0], "tiling": list(best[1]), "block_us": best[2], "tail_us": best[3],
             "gbs": bytes_per_launch / (best[3] * 1e-6) / 1e9,
             "all": [{"index": i, "tiling": list(t), "block_us": b, "tail_us": us} for i, t, b, us in res]}
    if write:
        d = load_cache()
        d[key(B, L, C)] = entry
        save_cache(d)
    return entry


def tuned(ctx, method: int, L: int, B: int, C: int) -> cv.TANConvolution:
    """A TANConvolution initialised and set to the cached best tiling, if any."""
    conv = cv.TANConvolution(ctx)
    rc = conv.Init(method, L, B, C)
    if rc != cv.AMF_OK:
        raise cv.TANError(rc, "Init")
    e = load_cache().get(key(B, L, C))
    if e is not None:
        conv.tiling(int(e["index"]))
    return conv



def tune_nu(ctx, C, L, B0, max_blocks=(1024, 2048, 4096, 8192), mids=(1, 2), spectrum=0, periods=2):
    """Times candidate schedules over whole periods of the largest level and
    returns them sorted by mean block time (device-resident input)."""
    import torch

    res = []
    g = np.random.Generator(np.random.PCG64(20261203 + 40))
    for mb in max_blocks:
        for mid in mids:
            lv = nupols.schedule(L, B0, mb)
            if mid == 1 and len(lv) > 2:
                # single partitions in the middle levels, the first level keeps two
                lv = [lv[0]] + [(b, 1) for b, _ in lv[1:-1]] + [lv[-1]]
                off = sum(b * k for b, k in lv[:-1])
                lv[-1] = (lv[-1][0], -(-(L - off) // lv[-1][0]))
            try:
                nu = nupols.NonUniform(ctx, C, L, lv, spectrum)
            except cv.TANError:
                continue
            period = lv[-1][0] // B0
            n = period * periods
            x = torch.from_numpy(g.uniform(-1, 1, (C, B0 * n)).astype(np.float32)).cuda()
            y = torch.zeros_like(x)
            st = torch.cuda.ExternalStream(nu.stream())
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
            for k in range(n):
                ev[k][0].record(st)
                nu.process_device(x.data_ptr() + k * B0 * 4, y.data_ptr() + k * B0 * 4, B0 * n)
                ev[k][1].record(st)
            nu.synchronize()
            ms = [a.elapsed_time(b) for a, b in ev]
            res.append({"levels": lv, "mean_ms": float(np.mean(ms[period:])), "max_ms": float(np.max(ms[period:])),
                        "tail_bytes_per_block": nu.info()["tail_bytes_per_block"]})
            nu.release()
            del x, y
    res.sort(key=lambda r: r["mean_ms"])
    return res


def nu_candidates(L, B0, max_blocks=(1024, 2048, 4096, 8192, 16384), mids=(1, 2)):
    """Level schedules the non-uniform search tries: the default doubling ladder
    (two partitions per size) up to each maximum block, and the same ladder
    with one partition in the middle levels."""
    out = []
    for mb in max_blocks:
        if mb < B0:
            continue
        for mid in mids:
            lv = nupols.schedule(L, B0, mb)
            if mid == 1 and len(lv) > 2:
                lv = [lv[0]] + [(b, 1) for b, _ in lv[1:-1]] + [lv[-1]]
                off = sum(b * k for b, k in lv[:-1])
                if any(sum(b * k for b, k in lv[:i]) < lv[i][0] for i in range(1, len(lv))):
                    continue  # a level would start before its block
                lv[-1] = (lv[-1][0], -(-(L - off) // lv[-1][0]))
            if lv not in out:
                out.append(lv)
    return out


def tune_nu_engine(ctx, C, L, B0, max_blocks=(1024, 2048, 4096, 8192, 16384), mids=(1, 2), spectrum=0,
                   items=(16, 32), periods=2):
    """Times every candidate schedule (nu_candidates) with every work-item size
    as one non-uniform engine session of C channels: CUDA events around each
    block launch (device rows), over `periods` periods of the largest level
    after one period of warm-up. Returns the results sorted by mean block time."""
    import torch

    from . import engine as eng

    res = []
    g = np.random.Generator(np.random.PCG64(20261203 + 41))
    h = (g.standard_normal((C, L)) * 1e-3).astype(np.float32)
    for lv in nu_candidates(L, B0, max_blocks, mids):
        period = lv[-1][0] // B0
        n = period * (periods + 1)
        x = torch.from_numpy(g.uniform(-1, 1, (C, B0 * n)).astype(np.float32)).cuda()
        y = torch.zeros_like(x)
        for q in items:
            e = eng.Engine(ctx, B0, spectrum, budget_bytes=eng.session_bytes(B0, C, L, lv, spectrum, q),
                           max_channels=C, partitions_per_item=q)
            rc, s = e.open_session_nu(C, L, lv)
            if rc != AMF_OK:
                e.release()
                continue
            assert s.update_response_td(h, block_until_ready=True) == AMF_OK
            st = torch.cuda.ExternalStream(e.stream())
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
            for k in range(n):
                ev[k][0].record(st)
                assert e.process_device(x.data_ptr() + k * B0 * 4, y.data_ptr() + k * B0 * 4, B0 * n) == AMF_OK
                ev[k][1].record(st)
            e.synchronize()
            ms = [a.elapsed_time(b) for a, b in ev][period:]
            res.append({"levels": lv, "partitions_per_item": q, "mean_ms": float(np.mean(ms)),
                        "p99_ms": float(np.percentile(ms, 99)), "max_ms": float(np.max(ms)),
                        "block_bytes": e.info()["block_bytes"]})
            e.release()
        del x, y
    res.sort(key=lambda r: r["mean_ms"])
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--block", type=int, default=512)
    ap.add_argument("--length", type=int, default=65536)
    ap.add_argument("--channels", type=int, default=64)
    a = ap.parse_args()
    ctx = cv.TANContext(0)
    e = tune(ctx, a.block, a.length, a.channels)
    print(json.dumps({key(a.block, a.length, a.channels): e}))


if __name__ == "__main__":
    main()
