"""Python mirror of the batched engine (tanb_engine_* in include/tanb.h).

A session is the equivalent of one TANConvolution object (C channels, IR
length L); every open session advances by one block per `process()` call, all
of them in one head and one tail launch. I/O goes through the engine's pinned
host buffers, exposed here as numpy views shaped (max_channels, block).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .convolution import AMF_OK, TANContext, TANError, lib

SPECTRUM_FP32 = 0
SPECTRUM_FP16 = 1
SPECTRUM_BF16 = 2
SPECTRUM_FP24 = 3  # IR spectra and delay line in 24 bits (engine only)


def session_bytes(block: int, channels: int, ir_length: int, levels=None, spectrum: int = SPECTRUM_FP32,
                  partitions_per_item: int = 0) -> int:
    """Device bytes a session takes from an engine's budget (host arithmetic,
    tanb_engine_session_bytes): uniform when levels is None, else the
    non-uniform schedule [(block, partitions), ...]."""
    nl = len(levels) if levels else 0
    blocks = (ctypes.c_uint32 * max(1, nl))(*[b for b, _ in (levels or [])])
    parts = (ctypes.c_uint32 * max(1, nl))(*[k for _, k in (levels or [])])
    out = ctypes.c_uint64(0)
    rc = lib().tanb_engine_session_bytes(block, spectrum, partitions_per_item, channels, ir_length, nl,
                                         blocks if nl else None, parts if nl else None, ctypes.byref(out))
    if rc != AMF_OK:
        raise TANError(rc, "tanb_engine_session_bytes")
    return out.value


class Session:
    def __init__(self, engine: "Engine", sid: int, first_slot: int, channels: int, ir_length: int):
        self.engine, self.id, self.first_slot = engine, sid, first_slot
        self.channels, self.ir_length = channels, ir_length

    @property
    def slots(self) -> slice:
        return slice(self.first_slot, self.first_slot + self.channels)

    def update_response_td(self, ir: np.ndarray, block_until_ready: bool = False) -> int:
        """New IR for every channel of the session; with block_until_ready the
        swap lands on the next block, otherwise on the first block after the
        transform (done on the engine's update stream) has finished."""
        ir = np.ascontiguousarray(ir, dtype=np.float32)
        rows = (ctypes.c_void_p * self.channels)(*[ir[c].ctypes.data for c in range(self.channels)])
        return lib().tanb_engine_update_response_td(self.engine._h, self.id, rows, ir.shape[1],
                                                    1 if block_until_ready else 0)

    def update_response_td_device(self, ir, block_until_ready: bool = False) -> int:
        """IR rows resident on the device: a (channels, n) CUDA tensor."""
        base, stride = ir.data_ptr(), ir.stride(0) * ir.element_size()
        rows = (ctypes.c_void_p * self.channels)(*[base + c * stride for c in range(self.channels)])
        return lib().tanb_engine_update_response_td_device(self.engine._h, self.id, rows, ir.shape[1],
                                                           1 if block_until_ready else 0)

    def state(self) -> dict:
        out = (ctypes.c_int64 * 3)()
        lib().tanb_engine_session_state(self.engine._h, self.id, out)
        return {"blocks": out[0], "last_swap_block": out[1], "staged": bool(out[2])}

    def snapshot(self):
        """(AMF_RESULT, uint8 array): the session's state, for
        Engine.open_session_restore on an engine with the same block, spectrum
        and partitions per item (uniformly partitioned sessions)."""
        n = ctypes.c_uint64(0)
        rc = lib().tanb_engine_session_snapshot_bytes(self.engine._h, self.id, ctypes.byref(n))
        if rc != AMF_OK:
            return rc, None
        buf = np.empty(n.value, np.uint8)
        rc = lib().tanb_engine_session_snapshot(self.engine._h, self.id, buf.ctypes.data, n.value)
        return rc, (buf if rc == AMF_OK else None)

    def close(self) -> int:
        return lib().tanb_engine_close_session(self.engine._h, self.id)


class Engine:
    def __init__(self, ctx: TANContext, block: int, spectrum: int = SPECTRUM_FP32, budget_bytes: int = 1 << 30,
                 max_channels: int = 1024, partitions_per_item: int = 32):
        h = ctypes.c_void_p()
        rc = lib().tanb_engine_create(ctx._h, block, spectrum, budget_bytes, max_channels, partitions_per_item,
                                      ctypes.byref(h))
        if rc != AMF_OK:
            raise TANError(rc, "tanb_engine_create")
        self._h = h
        self._ctx = ctx
        self.block = block
        self.max_channels = max_channels
        pin = ctypes.POINTER(ctypes.c_float)()
        pout = ctypes.POINTER(ctypes.c_float)()
        lib().tanb_engine_io(h, ctypes.byref(pin), ctypes.byref(pout))
        n = max_channels * block
        self.inp = np.ctypeslib.as_array(pin, shape=(n,)).reshape(max_channels, block)
        self.out = np.ctypeslib.as_array(pout, shape=(n,)).reshape(max_channels, block)

    def release(self):
        if self._h:
            lib().tanb_engine_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def open_session(self, channels: int, ir_length: int):
        """Returns (AMF_RESULT, Session or None)."""
        sid = ctypes.c_int32(0)
        first = ctypes.c_uint32(0)
        rc = lib().tanb_engine_open_session(self._h, channels, ir_length, ctypes.byref(sid), ctypes.byref(first))
        if rc != AMF_OK:
            return rc, None
        return rc, Session(self, sid.value, first.value, channels, ir_length)

    def open_session_restore(self, snapshot):
        """Opens a session from Session.snapshot(); returns (AMF_RESULT, Session or None)."""
        buf = np.ascontiguousarray(snapshot, dtype=np.uint8)
        sid = ctypes.c_int32(0)
        first = ctypes.c_uint32(0)
        rc = lib().tanb_engine_open_session_restore(self._h, buf.ctypes.data, buf.size, ctypes.byref(sid),
                                                    ctypes.byref(first))
        if rc != AMF_OK:
            return rc, None
        channels, ir_length = (int(v) for v in np.frombuffer(buf[20:28].tobytes(), np.uint32))
        return rc, Session(self, sid.value, first.value, channels, ir_length)

    def open_session_nu(self, channels: int, ir_length: int, levels):
        """Non-uniformly partitioned session; levels = [(block, partitions), ...]
        with levels[0][0] == the engine block. Returns (AMF_RESULT, Session or None)."""
        nl = len(levels)
        blocks = (ctypes.c_uint32 * nl)(*[b for b, _ in levels])
        parts = (ctypes.c_uint32 * nl)(*[k for _, k in levels])
        sid = ctypes.c_int32(0)
        first = ctypes.c_uint32(0)
        rc = lib().tanb_engine_open_session_nu(self._h, channels, ir_length, nl, blocks, parts, ctypes.byref(sid),
                                               ctypes.byref(first))
        if rc != AMF_OK:
            return rc, None
        return rc, Session(self, sid.value, first.value, channels, ir_length)

    def write_input(self, first_slot: int, x: np.ndarray) -> int:
        """Copies the first `block` samples of each row of x (float32, C-contiguous
        rows) into the input buffer at slots first_slot, first_slot + 1, ..."""
        if x.dtype != np.float32 or not x.flags.c_contiguous or x.ndim != 2:
            raise TypeError("x must be a C-contiguous float32 (rows, samples) array")
        return lib().tanb_engine_write_input(self._h, first_slot, x.ctypes.data, x.shape[0], x.shape[1])

    def process(self) -> int:
        return lib().tanb_engine_process(self._h)

    def process_device(self, d_in: int, d_out: int, ld: int = 0) -> int:
        return lib().tanb_engine_process_device(self._h, d_in, d_out, ld)

    def synchronize(self) -> int:
        return lib().tanb_engine_synchronize(self._h)

    def stream(self) -> int:
        return lib().tanb_engine_stream(self._h) or 0

    def info(self) -> dict:
        out = (ctypes.c_int64 * 8)()
        lib().tanb_engine_info(self._h, out)
        keys = ("sessions", "channels", "slot_hwm", "item_hwm", "arena_bytes", "budget", "block_bytes",
                "tail_grid")
        return dict(zip(keys, list(out)))

    def block_times(self) -> dict:
        """Host microseconds of the last process() call, by part; max_us is
        the longest call since the previous read."""
        us = (ctypes.c_double * 8)()
        lib().tanb_engine_block_times(self._h, us)
        keys = ("lock_us", "commit_us", "graph_build_us", "launch_us", "wait_us", "total_us", "max_us",
                "graph_builds")
        return dict(zip(keys, list(us)))

    def profile(self, enable: bool) -> int:
        return lib().tanb_engine_profile(self._h, 1 if enable else 0)

    def profile_read(self) -> dict:
        counts = (ctypes.c_int64 * 4)()
        ms = (ctypes.c_double * 2)()
        lib().tanb_engine_profile_read(self._h, counts, ms)
        return {"blocks": counts[0], "commits": counts[1], "ir_updates": counts[2], "timed": counts[3],
                "block_ms": ms[0]}
