"""TEST INFRASTRUCTURE ONLY -- the FP64 oracle.

Only tests/, the smoke check and bench.py's CPU legs import this module, as the
checker; the product path (libtanb.so and the tan_b200 package) never does.

Double-precision statement of what TrueAudio Next's TANConvolution computes for
one stream of blocks (tan/tanlibrary/include/TrueAudioNext.h:125-250):

* steady state: output block k is samples [kB, kB+B) of the linear convolution
  of the channel's input with its active impulse response (zero extra latency,
  tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:2380-2535);
* an IR swap takes effect on the first block processed after UpdateResponseTD
  returns and that block is a linear crossfade over one block,
  out[i] = new[i] * (i/B) + old[i] * ((B-i)/B)  (ConvolutionImpl.cpp:877, 1392-1408),
  where new and old are the outputs of each IR over the full input history;
* the initial IR is all zeros (slot state at construction, ConvolutionImpl.cpp:115);
* a flush before block f discards the history before sample fB
  (ConvolutionImpl.cpp:1261-1351, intended semantics).
"""
from __future__ import annotations

import numpy as np


def _nextpow2(n: int) -> int:
    p = 1
    while p < n:
        p <<= 1
    return p


def conv_fp64(x: np.ndarray, h: np.ndarray) -> np.ndarray:
    """First len(x) samples of the linear convolution x * h, in float64 (FFT)."""
    x = np.asarray(x, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    T = x.shape[-1]
    if h.size == 0 or T == 0:
        return np.zeros(T)
    n = _nextpow2(T + h.size - 1)
    y = np.fft.irfft(np.fft.rfft(x, n) * np.fft.rfft(h, n), n)
    return y[:T]


def direct_fp64(x: np.ndarray, h: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Direct sums y[n] = sum_k h[k] x[n-k] at the given output indices, float64."""
    x = np.asarray(x, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    out = np.empty(len(idx))
    for j, n in enumerate(idx):
        k = np.arange(min(n, h.size - 1) + 1)
        out[j] = np.dot(h[k], x[n - k])
    return out


def stream_fp64(x: np.ndarray, B: int, ir_events, flush_events=None) -> np.ndarray:
    """Expected output of a block stream with IR swaps and flushes, float64.

    x            (C, T) input, T a multiple of B
    ir_events    list of (block k, {channel: ir}) -- UpdateResponseTD before block k
    flush_events list of (block k, [channels]) -- history cleared before block k
    """
    x = np.asarray(x, dtype=np.float64)
    C, T = x.shape
    nb = T // B
    y = np.zeros((C, nb * B))
    flush_events = flush_events or []
    for c in range(C):
        versions = [(-1, np.zeros(1))]  # (first block, ir); the zero IR predates block 0
        for k, irs in sorted(ir_events, key=lambda e: e[0]):
            if c in irs:
                h = np.asarray(irs[c], dtype=np.float64)
                if versions[-1][0] == k:  # replaced before it took effect
                    versions[-1] = (k, h)
                else:
                    versions.append((k, h))
        epochs = sorted({0} | {k for k, chans in flush_events if c in chans})
        cache = {}

        def full(ep_start, v):
            key = (ep_start, v)
            if key not in cache:
                xe = x[c].copy()
                xe[: ep_start * B] = 0.0
                cache[key] = conv_fp64(xe, versions[v][1])
            return cache[key]

        w1 = np.arange(B) / B
        w2 = (B - np.arange(B)) / B
        for k in range(nb):
            ep = max(e for e in epochs if e <= k)
            v = max(i for i, (k0, _) in enumerate(versions) if k0 <= k)
            sl = slice(k * B, (k + 1) * B)
            if versions[v][0] == k:
                y[c, sl] = full(ep, v)[sl] * w1 + full(ep, v - 1)[sl] * w2
            else:
                y[c, sl] = full(ep, v)[sl]
    return y


def exp_decay_ir(rng: np.random.Generator, n: int, rt60_s: float, fs: int = 48000) -> np.ndarray:
    """Gaussian noise times exp(-ln(1000) n / (RT60 fs)), unit L2 norm (float32)."""
    t = np.arange(n, dtype=np.float64)
    h = rng.standard_normal(n) * np.exp(-np.log(1000.0) * t / (rt60_s * fs))
    h /= np.linalg.norm(h)
    return h.astype(np.float32)


def error_db(y: np.ndarray, ref: np.ndarray) -> float:
    """20 log10(rms(y - ref) / rms(ref))."""
    ref = np.asarray(ref, dtype=np.float64)
    d = np.asarray(y, dtype=np.float64) - ref
    r = np.sqrt(np.mean(ref * ref))
    e = np.sqrt(np.mean(d * d))
    if e == 0.0:
        return -np.inf
    return float(20.0 * np.log10(e / r))
