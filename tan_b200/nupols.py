"""Python mirror of the non-uniformly partitioned convolution (tanb_nu_* in
include/tanb.h): levels of growing block size along the IR, zero added latency."""
from __future__ import annotations

import ctypes

import numpy as np

from .convolution import AMF_OK, TANError, lib


def schedule(ir_length: int, base_block: int, max_block: int):
    """Default level schedule: [(block, partitions), ...]."""
    n = ctypes.c_uint32(0)
    blocks = (ctypes.c_uint32 * 16)()
    parts = (ctypes.c_uint32 * 16)()
    rc = lib().tanb_nu_schedule(ir_length, base_block, max_block, ctypes.byref(n), blocks, parts)
    if rc != AMF_OK:
        raise TANError(rc, "tanb_nu_schedule")
    return [(blocks[i], parts[i]) for i in range(n.value)]


def coverage(levels) -> int:
    return sum(b * k for b, k in levels)


class NonUniform:
    def __init__(self, ctx, channels: int, ir_length: int, levels, spectrum: int = 0):
        nl = len(levels)
        blocks = (ctypes.c_uint32 * nl)(*[b for b, _ in levels])
        parts = (ctypes.c_uint32 * nl)(*[k for _, k in levels])
        h = ctypes.c_void_p()
        rc = lib().tanb_nu_create(ctx._h, channels, ir_length, nl, blocks, parts, spectrum, ctypes.byref(h))
        if rc != AMF_OK:
            raise TANError(rc, "tanb_nu_create")
        self._h, self._ctx = h, ctx
        self.channels, self.ir_length, self.levels = channels, ir_length, list(levels)
        self.block = levels[0][0]
        pin = ctypes.POINTER(ctypes.c_float)()
        pout = ctypes.POINTER(ctypes.c_float)()
        lib().tanb_nu_io(h, ctypes.byref(pin), ctypes.byref(pout))
        n = channels * self.block
        self.inp = np.ctypeslib.as_array(pin, shape=(n,)).reshape(channels, self.block)
        self.out = np.ctypeslib.as_array(pout, shape=(n,)).reshape(channels, self.block)

    def release(self):
        if self._h:
            lib().tanb_nu_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def set_response(self, ir: np.ndarray) -> int:
        ir = np.ascontiguousarray(ir, dtype=np.float32)
        rows = (ctypes.c_void_p * self.channels)(*[ir[c].ctypes.data for c in range(self.channels)])
        return lib().tanb_nu_set_response(self._h, rows, ir.shape[1])

    def process(self) -> int:
        return lib().tanb_nu_process(self._h)

    def process_device(self, d_in: int, d_out: int, ld: int = 0) -> int:
        return lib().tanb_nu_process_device(self._h, d_in, d_out, ld)

    def synchronize(self) -> int:
        return lib().tanb_nu_synchronize(self._h)

    def stream(self) -> int:
        return lib().tanb_nu_stream(self._h) or 0

    def info(self) -> dict:
        out = (ctypes.c_int64 * 6)()
        lib().tanb_nu_info(self._h, out)
        return dict(zip(("channels", "block", "levels", "device_bytes", "tail_bytes_per_block", "blocks"), out))

    def run(self, x: np.ndarray) -> np.ndarray:
        """Processes x (channels, T), T a multiple of the base block, through the host buffers."""
        C, T = x.shape
        B = self.block
        y = np.zeros_like(x, dtype=np.float32)
        for k in range(T // B):
            self.inp[:] = x[:, k * B:(k + 1) * B]
            rc = self.process()
            if rc != AMF_OK:
                raise TANError(rc, "tanb_nu_process")
            y[:, k * B:(k + 1) * B] = self.out
        return y
