"""TEST INFRASTRUCTURE ONLY -- ctypes binding of the oracle's C++ restatement
of TAN's CPU uniformly-partitioned convolution (oracle/tan_cpu_ref.cpp).

Used by tests/, the smoke check and bench.py's CPU legs as the checker and the
timed CPU baseline; never by the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtanref.so")
_lib = None


def build() -> str:
    """Compile libtanref.so with the oracle's Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, i32, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
        fpp = ctypes.POINTER(ctypes.c_void_p)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.tanref_create.restype = vp
        L.tanref_create.argtypes = [i32, i32, i32, i32]
        L.tanref_destroy.argtypes = [vp]
        L.tanref_partitions.argtypes = [vp]
        L.tanref_partitions.restype = i32
        L.tanref_update_td.argtypes = [vp, fpp, sz, u32p]
        L.tanref_update_td.restype = i32
        L.tanref_process.argtypes = [vp, fpp, fpp, sz, u32p, ctypes.POINTER(sz)]
        L.tanref_process.restype = i32
        L.tanref_next_free_channel.argtypes = [vp, u32p, u32p]
        L.tanref_next_free_channel.restype = i32
        L.tanref_td_create.restype = vp
        L.tanref_td_create.argtypes = [i32, i32]
        L.tanref_td_destroy.argtypes = [vp]
        L.tanref_td_process_direct.restype = i32
        L.tanref_td_process_direct.argtypes = [vp, fpp, fpp, fpp, sz, ctypes.POINTER(sz),
                                               ctypes.POINTER(ctypes.c_int32)]
        fp = ctypes.c_void_p
        L.tanref_rfft.argtypes = [i32, fp, fp, fp]
        s16p = ctypes.POINTER(ctypes.c_int16)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.tanref_convert_s16_f32.argtypes = [s16p, sz, sz, fp, sz, ctypes.c_float]
        L.tanref_convert_s16_f32.restype = None
        for name in ("tanref_convert_f32_s16", "tanref_convert_f32_s16_dev"):
            getattr(L, name).argtypes = [fp, sz, sz, s16p, sz, ctypes.c_float, i32p]
            getattr(L, name).restype = None
        L.tanref_mix.argtypes = [fpp, i32, sz, fp]
        L.tanref_mix.restype = None
        L.tanref_mix_dev.argtypes = [fp, sz, i32, sz, fp]
        L.tanref_mix_dev.restype = None
        L.tanref_room_response.argtypes = [fp, fp, fp, i32, i32, i32, fp, fp, i32, i32, fp, fp]
        L.tanref_room_response.restype = ctypes.c_long
        L.tanref_irfft.argtypes = [i32, fp, fp, fp]
        _lib = L
    return _lib


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _flags(flags, C):
    if flags is None:
        return None
    f = np.ascontiguousarray(np.asarray(flags, dtype=np.uint32).reshape(C))
    return f, f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


class RefConvolution:
    """Mirror of TANConvolution (Init / UpdateResponseTD / Process /
    GetNextFreeChannel) over the restatement; arrays are (channels, samples)."""

    def __init__(self, length: int, block: int, channels: int, threads: int = 1):
        self.L, self.B, self.C = length, block, channels
        self._h = lib().tanref_create(length, block, channels, threads)
        if not self._h:
            raise ValueError("invalid oracle configuration")

    def close(self):
        if self._h:
            lib().tanref_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def partitions(self) -> int:
        return lib().tanref_partitions(self._h)

    def update_response_td(self, ir: np.ndarray, flags=None) -> int:
        ir = np.ascontiguousarray(ir, dtype=np.float32)
        rows = [np.ascontiguousarray(ir[c]) for c in range(self.C)]
        fl = _flags(flags, self.C)
        return lib().tanref_update_td(self._h, _ptrs(rows), ir.shape[1], fl[1] if fl else None)

    def process(self, x: np.ndarray, flags=None, out: np.ndarray | None = None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[1]
        if out is None:
            out = np.zeros_like(x)
        rows_in = [x[c] for c in range(self.C)]
        rows_out = [out[c] for c in range(self.C)]
        fl = _flags(flags, self.C)
        done = ctypes.c_size_t(0)
        rc = lib().tanref_process(self._h, _ptrs(rows_in), _ptrs(rows_out), n,
                                  fl[1] if fl else None, ctypes.byref(done))
        return rc, out, done.value

    def next_free_channel(self, flags=None):
        idx = ctypes.c_uint32(0)
        fl = _flags(flags, self.C)
        rc = lib().tanref_next_free_channel(self._h, ctypes.byref(idx), fl[1] if fl else None)
        return rc, idx.value


class RefTimeDomain:
    """Mirror of TANConvolution::ProcessDirect for TIME_DOMAIN over the restatement."""

    def __init__(self, length: int, channels: int):
        self.L, self.C = length, channels
        self._h = lib().tanref_td_create(length, channels)
        if not self._h:
            raise ValueError("invalid oracle configuration")

    def close(self):
        if self._h:
            lib().tanref_td_destroy(self._h)
            self._h = None

    __del__ = close

    def process_direct(self, ir: np.ndarray, x: np.ndarray, nz=None):
        ir = np.ascontiguousarray(ir, dtype=np.float32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros_like(x)
        nzp = None
        if nz is not None:
            nzk = np.ascontiguousarray(np.asarray(nz, dtype=np.int32))
            nzp = nzk.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        done = ctypes.c_size_t(0)
        rc = lib().tanref_td_process_direct(self._h, _ptrs([ir[c] for c in range(self.C)]),
                                            _ptrs([x[c] for c in range(self.C)]),
                                            _ptrs([out[c] for c in range(self.C)]), x.shape[1],
                                            ctypes.byref(done), nzp)
        return rc, out, done.value


def rfft(x: np.ndarray):
    x = np.ascontiguousarray(x, dtype=np.float32)
    N = x.size
    re = np.zeros(N // 2 + 1, np.float32)
    im = np.zeros(N // 2 + 1, np.float32)
    lib().tanref_rfft(N, x.ctypes.data, re.ctypes.data, im.ctypes.data)
    return re, im


def irfft(re: np.ndarray, im: np.ndarray):
    re = np.ascontiguousarray(re, dtype=np.float32)
    im = np.ascontiguousarray(im, dtype=np.float32)
    N = 2 * (re.size - 1)
    y = np.zeros(N, np.float32)
    lib().tanref_irfft(N, re.ctypes.data, im.ctypes.data, y.ctypes.data)
    return y


# --- TANConverter / TANMixer restatements --------------------------------------


def _span(a: np.ndarray, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(ctypes.POINTER(np.ctypeslib.as_ctypes_type(dtype)))


def convert_s16_f32(x: np.ndarray, gain: float, in_step: int = 1, n: int | None = None) -> np.ndarray:
    """short -> float (ConverterImpl.cpp:217-246) of samples x[0], x[in_step], ..."""
    x, px = _span(x, np.int16)
    n = (x.size + in_step - 1) // in_step if n is None else n
    y = np.zeros(n, np.float32)
    lib().tanref_convert_s16_f32(px, in_step, n, y.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 1, gain)
    return y


def convert_f32_s16(x: np.ndarray, gain: float, in_step: int = 1, n: int | None = None, device: bool = False):
    """float -> short; (output, clipped). device=False: the CPU overload
    (ConverterImpl.cpp:287-408); device=True: the OpenCL kernel (Converter.cl:97-120)."""
    x, px = _span(x, np.float32)
    n = (x.size + in_step - 1) // in_step if n is None else n
    y = np.zeros(n, np.int16)
    clip = ctypes.c_int32(0)
    fn = lib().tanref_convert_f32_s16_dev if device else lib().tanref_convert_f32_s16
    fn(px, in_step, n, y.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)), 1, gain, ctypes.byref(clip))
    return y, bool(clip.value)


def mix(x: np.ndarray, device: bool = False) -> np.ndarray:
    """Sum over channels of x (channels, n) in channel order: MixerImpl.cpp:226-250
    (device=False) or Mixer.cl:26-41 (device=True)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    C, n = x.shape
    y = np.zeros(n, np.float32)
    py = y.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    if device:
        lib().tanref_mix_dev(x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, C, n, py)
    else:
        lib().tanref_mix(_ptrs([x[c] for c in range(C)]), C, n, py)
    return y


# --- Room response producer restatement -----------------------------------------


def room_response(room, source, ears, rate: int, length: int, low_pass, high_pass, flags: int = 0,
                  max_bounces: int = 0):
    """Left / right IRs of a shoebox room (the GPU path of
    TrueAudioVR::generateRoomResponse). room: (width, height, length, damp left,
    right, top, bottom, front, back); source: (x, y, z); ears: (head x, y, z,
    ear spacing, yaw, pitch, roll). Returns (left, right, images per ear)."""
    fp = ctypes.POINTER(ctypes.c_float)
    r = np.ascontiguousarray(room, np.float32)
    s = np.ascontiguousarray(source, np.float32)
    e = np.ascontiguousarray(ears, np.float32)
    lp = np.ascontiguousarray(low_pass, np.float32)
    hp = np.ascontiguousarray(high_pass, np.float32)
    left = np.zeros(length, np.float32)
    right = np.zeros(length, np.float32)
    n = lib().tanref_room_response(r.ctypes.data_as(fp), s.ctypes.data_as(fp), e.ctypes.data_as(fp), rate, length,
                                   lp.size, lp.ctypes.data_as(fp), hp.ctypes.data_as(fp), flags, max_bounces,
                                   left.ctypes.data_as(fp), right.ctypes.data_as(fp))
    return left, right, int(n)


def simple_head_filters(ear_spacing: float = 0.16, n: int = 64, rate: int = 48000):
    """The head-shadow low-pass / complementary high-pass pair of
    TrueAudioVR::generateSimpleHeadRelatedTransform (TrueAudioVR.cpp:361-411),
    with numpy's FFT in place of TAN's: a test input for the room producer."""
    corner = np.float32(343.0 / (1.10 * ear_spacing))
    f = np.array([(j // 2) / (n * (1.0 / rate)) for j in range(n)], np.float32)
    d = corner / (corner + f)
    spec = np.fft.fft(np.eye(1, n, 0)[0]) * d
    low = np.real(np.fft.ifft(spec)).astype(np.float32)
    high = -low
    high[0] += 1.0
    return low, high.astype(np.float32)
