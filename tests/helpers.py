"""Shared helpers for the tests: seeded synthetic inputs and block-stream drivers."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import fp64

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def noise(g, C, T, scale=1.0):
    return (g.uniform(-1.0, 1.0, (C, T)) * scale).astype(np.float32)


def irs(g, C, L, rt60=(0.3, 0.3)):
    return np.stack([fp64.exp_decay_ir(g, L, float(g.uniform(*rt60))) for _ in range(C)])


def golden_taps():
    with open(os.path.join(GOLDEN, "testresponse_taps.json")) as f:
        return json.load(f)


def delta_irs(length=None):
    """The reference's testresponse.wav delta IRs as float32 arrays."""
    g = golden_taps()
    n = length or g["length"]
    h = np.zeros((len(g["channels"]), n), np.float32)
    for c, taps in enumerate(g["channels"]):
        for t in taps:
            h[c, t["index"]] = np.float32(t["value"])
    return h


def pulsetrain(C=2):
    x = np.load(os.path.join(GOLDEN, "pulsetrainS_head.npy")).astype(np.float32) / 32768.0
    return np.ascontiguousarray(x[:C])


def run_stream(conv, x, B, events=None, flags_per_block=None, per_call_blocks=1):
    """Drives conv (GPU mirror or oracle) over x block by block.

    events: {block: (ir array (C, n), flags or None)} applied before that block.
    flags_per_block: optional list of per-channel flag arrays.
    Returns (outputs, list of return codes).
    """
    C, T = x.shape
    nb = T // B
    y = np.zeros((C, nb * B), np.float32)
    codes = []
    events = events or {}
    k = 0
    while k < nb:
        if k in events:
            ir, fl = events[k]
            rc = conv.update_response_td(ir, fl) if hasattr(conv, "update_response_td") else conv.UpdateResponseTD(
                np.ascontiguousarray(ir, dtype=np.float32), ir.shape[1], fl)
            assert rc == 0, rc
        step = 1 if flags_per_block is not None else per_call_blocks
        step = min(step, nb - k)
        while step > 1 and any(j in events for j in range(k + 1, k + step)):
            step -= 1
        xs = np.ascontiguousarray(x[:, k * B:(k + step) * B])
        ys = np.ascontiguousarray(y[:, k * B:(k + step) * B])
        fl = flags_per_block[k] if flags_per_block is not None else None
        if hasattr(conv, "process"):
            rc, ys, done = conv.process(xs, fl, ys)
        else:
            rc, done = conv.Process(xs, ys, step * B, fl)
        codes.append(rc)
        if rc == 0:
            assert done == step * B, (done, step * B)
        y[:, k * B:(k + step) * B] = ys
        k += step
    return y, codes


def rel_err(y, ref):
    """max |y - ref| / rms(ref) over all samples."""
    ref = np.asarray(ref, np.float64)
    r = np.sqrt(np.mean(ref * ref))
    return float(np.max(np.abs(np.asarray(y, np.float64) - ref)) / r)
