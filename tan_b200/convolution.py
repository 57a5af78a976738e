"""Python mirror of amf::TANConvolution over the C ABI in libtanb.so.

Method names, argument meaning and AMF_RESULT return codes follow
tan/tanlibrary/include/TrueAudioNext.h:125-253; sample buffers are numpy arrays
shaped (channels, samples) (or any sequence of per-channel 1-D float32 arrays)
for the host overloads and CUDA tensors (anything with .data_ptr()) for the
device overloads. Every call goes to the CUDA path; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtanb.so")

# AMF_RESULT (amf/public/include/core/Result.h:43-125)
AMF_OK = 0
AMF_FAIL = 1
AMF_UNEXPECTED = 2
AMF_INVALID_ARG = 4
AMF_OUT_OF_RANGE = 5
AMF_OUT_OF_MEMORY = 6
AMF_INVALID_POINTER = 7
AMF_NOT_IMPLEMENTED = 9
AMF_NOT_SUPPORTED = 10
AMF_NOT_FOUND = 11
AMF_ALREADY_INITIALIZED = 12
AMF_NOT_INITIALIZED = 13
AMF_WRONG_STATE = 15
AMF_NO_DEVICE = 17
AMF_TAN_UNSUPPORTED_VERSION = 43

# TAN_CONVOLUTION_METHOD (TrueAudioNext.h:81-99)
TAN_CONVOLUTION_METHOD_FFT_OVERLAP_ADD = 0
TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_UNIFORM = 1
TAN_CONVOLUTION_METHOD_FFT_PARTITIONED_NONUNIFORM = 2
TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED = 3
TAN_CONVOLUTION_METHOD_FHT_UNIFORM_PARTITIONED = 4
TAN_CONVOLUTION_METHOD_FFT_UNIFORM_HEAD_TAIL = 5
TAN_CONVOLUTION_METHOD_FHT_UNIFORM_HEAD_TAIL = 6
TAN_CONVOLUTION_METHOD_TIME_DOMAIN = 7
TAN_CONVOLUTION_METHOD_FHT_NONUNIFORM_PARTITIONED = 8
TAN_CONVOLUTION_METHOD_FFT_NONUNIFORM_PARTITIONED = 9
TAN_CONVOLUTION_METHOD_USE_PROCESS_FINALIZE = 0x8000
TAN_CONVOLUTION_METHOD_USE_PROCESS_TAILTHREAD = 0xC000

# TAN_CONVOLUTION_CHANNEL_FLAG (TrueAudioNext.h:105-110)
TAN_CONVOLUTION_CHANNEL_FLAG_PROCESS = 0
TAN_CONVOLUTION_CHANNEL_FLAG_STOP_INPUT = 0x01
TAN_CONVOLUTION_CHANNEL_FLAG_FLUSH_STREAM = 0x02

# TAN_CONVOLUTION_OPERATION_FLAG (TrueAudioNext.h:116-120)
TAN_CONVOLUTION_OPERATION_FLAG_NONE = 0x00
TAN_CONVOLUTION_OPERATION_FLAG_BLOCK_UNTIL_READY = 0x01

TAN_FULL_VERSION = (1 << 48) | (3 << 32) | (1 << 16) | 1

# Every symbol include/tanb.h declares, with its ctypes signature.
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_u32 = ctypes.c_uint32
_sz = ctypes.c_size_t
_pp = ctypes.POINTER(ctypes.c_void_p)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_szp = ctypes.POINTER(ctypes.c_size_t)
SIGNATURES = {
    "tanb_create_context": (_i32, [ctypes.c_uint64, _i32, ctypes.POINTER(_vp)]),
    "tanb_context_release": (_i32, [_vp]),
    "tanb_create_convolution": (_i32, [_vp, ctypes.POINTER(_vp)]),
    "tanb_convolution_release": (_i32, [_vp]),
    "tanb_convolution_init": (_i32, [_vp, _u32, _u32, _u32, _u32]),
    "tanb_convolution_init_nu": (_i32, [_vp, _u32, _u32, _u32, _u32, _u32, _u32p, _u32p]),
    "tanb_convolution_terminate": (_i32, [_vp]),
    "tanb_convolution_update_response_td": (_i32, [_vp, _pp, _sz, _u32p, _u32]),
    "tanb_convolution_update_response_td_device": (_i32, [_vp, _pp, _sz, _u32p, _u32]),
    "tanb_convolution_update_response_fd": (_i32, [_vp, _pp, _sz, _u32p, _u32]),
    "tanb_convolution_process": (_i32, [_vp, _pp, _pp, _sz, _u32p, _szp]),
    "tanb_convolution_process_host_to_device": (_i32, [_vp, _pp, _pp, _sz, _u32p, _szp]),
    "tanb_convolution_process_device": (_i32, [_vp, _pp, _pp, _sz, _u32p, _szp]),
    "tanb_convolution_process_direct": (_i32, [_vp, _pp, _pp, _pp, _sz, _szp, ctypes.POINTER(ctypes.c_int32)]),
    "tanb_convolution_process_finalize": (_i32, [_vp]),
    "tanb_convolution_get_next_free_channel": (_i32, [_vp, _u32p, _u32p]),
    "tanb_convolution_synchronize": (_i32, [_vp]),
    "tanb_convolution_stream": (_vp, [_vp]),
    "tanb_convolution_info": (_i32, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "tanb_convolution_tiling": (_i32, [_vp, _i32, ctypes.POINTER(ctypes.c_int32)]),
    "tanb_convolution_profile": (_i32, [_vp, _i32]),
    "tanb_convolution_set_wait_limit": (_i32, [_vp, _i32]),
    "tanb_convolution_profile_read": (_i32, [_vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]),
    "tanb_engine_create": (_i32, [_vp, _u32, _u32, ctypes.c_uint64, _u32, _u32, ctypes.POINTER(_vp)]),
    "tanb_engine_release": (_i32, [_vp]),
    "tanb_engine_open_session": (_i32, [_vp, _u32, _u32, ctypes.POINTER(ctypes.c_int32), _u32p]),
    "tanb_engine_open_session_nu": (_i32, [_vp, _u32, _u32, _u32, _u32p, _u32p, ctypes.POINTER(ctypes.c_int32),
                                            _u32p]),
    "tanb_engine_close_session": (_i32, [_vp, _i32]),
    "tanb_engine_session_bytes": (_i32, [_u32, _u32, _u32, _u32, _u32, _u32, _u32p, _u32p,
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "tanb_engine_update_response_td": (_i32, [_vp, _i32, _pp, _sz, _u32]),
    "tanb_engine_update_response_td_device": (_i32, [_vp, _i32, _pp, _sz, _u32]),
    "tanb_engine_io": (_i32, [_vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)),
                              ctypes.POINTER(ctypes.POINTER(ctypes.c_float))]),
    "tanb_engine_write_input": (_i32, [_vp, _u32, _vp, _u32, _sz]),
    "tanb_engine_process": (_i32, [_vp]),
    "tanb_engine_process_device": (_i32, [_vp, _vp, _vp, _u32]),
    "tanb_engine_synchronize": (_i32, [_vp]),
    "tanb_engine_stream": (_vp, [_vp]),
    "tanb_engine_info": (_i32, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "tanb_engine_session_state": (_i32, [_vp, _i32, ctypes.POINTER(ctypes.c_int64)]),
    "tanb_engine_profile": (_i32, [_vp, _i32]),
    "tanb_engine_profile_read": (_i32, [_vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]),
    "tanb_engine_block_times": (_i32, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "tanb_convolution_call_times": (_i32, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "tanb_engine_session_snapshot_bytes": (_i32, [_vp, _i32, ctypes.POINTER(ctypes.c_uint64)]),
    "tanb_engine_session_snapshot": (_i32, [_vp, _i32, _vp, ctypes.c_uint64]),
    "tanb_engine_open_session_restore": (_i32, [_vp, _vp, ctypes.c_uint64, ctypes.POINTER(_i32),
                                                ctypes.POINTER(ctypes.c_uint32)]),
    "tanb_convolution_snapshot_bytes": (_i32, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "tanb_convolution_snapshot": (_i32, [_vp, _vp, ctypes.c_uint64]),
    "tanb_convolution_restore": (_i32, [_vp, _vp, ctypes.c_uint64]),
    "tanb_convolution_process_mix_pcm16": (_i32, [_vp, _pp, _sz, ctypes.c_float, _u32p, _u32, _pp, _sz,
                                                  ctypes.c_float, _sz, ctypes.POINTER(ctypes.c_int32), _szp]),
    "tanb_room_generator_create": (_i32, [_vp, _i32, ctypes.POINTER(_vp)]),
    "tanb_room_generator_release": (_i32, [_vp]),
    "tanb_room_response": (_i32, [_vp, _vp, _vp, _vp, _i32, _i32, _vp, _vp, _u32, _i32, _vp]),
    "tanb_room_images": (ctypes.c_int64, [_vp]),
    "tanb_room_generator_synchronize": (_i32, [_vp]),
    "tanb_room_generator_stream": (_vp, [_vp]),
    "tanb_converter_create": (_i32, [_vp, ctypes.POINTER(_vp)]),
    "tanb_converter_release": (_i32, [_vp]),
    "tanb_converter_short_to_float": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz, ctypes.c_float]),
    "tanb_converter_float_to_short": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz, ctypes.c_float,
                                             ctypes.POINTER(ctypes.c_int32)]),
    "tanb_converter_short_to_float_batch": (_i32, [_vp, _pp, _sz, _sz, _pp, _sz, ctypes.c_float, _i32]),
    "tanb_converter_float_to_short_batch": (_i32, [_vp, _pp, _sz, _sz, _pp, _sz, ctypes.c_float, _i32,
                                                   ctypes.POINTER(ctypes.c_int32)]),
    "tanb_converter_convert_device": (_i32, [_vp, _pp, _sz, _szp, _i32, _pp, _sz, _szp, _i32, _sz, ctypes.c_float,
                                             _i32, ctypes.POINTER(ctypes.c_int32)]),
    "tanb_converter_synchronize": (_i32, [_vp]),
    "tanb_converter_stream": (_vp, [_vp]),
    "tanb_mixer_create": (_i32, [_vp, _sz, _i32, ctypes.POINTER(_vp)]),
    "tanb_mixer_release": (_i32, [_vp]),
    "tanb_mixer_mix": (_i32, [_vp, _pp, _vp]),
    "tanb_mixer_mix_device": (_i32, [_vp, _pp, _vp]),
    "tanb_mixer_mix_device_strided": (_i32, [_vp, _vp, _vp, _sz]),
    "tanb_mixer_synchronize": (_i32, [_vp]),
    "tanb_mixer_stream": (_vp, [_vp]),
    "tanb_nu_schedule": (_i32, [_u32, _u32, _u32, _u32p, _u32p, _u32p]),
    "tanb_nu_create": (_i32, [_vp, _u32, _u32, _u32, _u32p, _u32p, _u32, ctypes.POINTER(_vp)]),
    "tanb_nu_release": (_i32, [_vp]),
    "tanb_nu_set_response": (_i32, [_vp, _pp, _sz]),
    "tanb_nu_io": (_i32, [_vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)),
                          ctypes.POINTER(ctypes.POINTER(ctypes.c_float))]),
    "tanb_nu_process": (_i32, [_vp]),
    "tanb_nu_process_device": (_i32, [_vp, _vp, _vp, _u32]),
    "tanb_nu_synchronize": (_i32, [_vp]),
    "tanb_nu_stream": (_vp, [_vp]),
    "tanb_nu_info": (_i32, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "tanb_convolve_no_alloc": (_i32, [_vp, _vp, _vp, _u32, _sz, _sz, _u32, _vp]),
    "tanb_stream_read": (_i32, [_vp, _sz, _vp, _u32, _u32, _vp]),
    "tanb_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libtanb.so; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m tan_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().tanb_last_error().decode()


class TANError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where} failed with AMF_RESULT {code}: {last_error()}")
        self.code = code


def _rows_host(buf, channels: int):
    """Per-channel float32 row pointers of a host buffer; returns (keepalive, ptr array)."""
    if isinstance(buf, np.ndarray) and buf.ndim == 2:
        if buf.dtype != np.float32 or not buf.flags.c_contiguous:
            raise TypeError("host buffers must be C-contiguous float32 (channels, samples)")
        if buf.shape[0] != channels:
            raise ValueError(f"expected {channels} channel rows, got {buf.shape[0]}")
        # row addresses computed at once (a view per row costs microseconds each)
        ptrs = np.uint64(buf.__array_interface__["data"][0]) + np.arange(channels, dtype=np.uint64) * np.uint64(
            buf.strides[0])
        return buf, (ctypes.c_void_p * channels).from_buffer_copy(ptrs.tobytes())
    rows = list(buf)
    for r in rows:
        if r is not None and (not isinstance(r, np.ndarray) or r.dtype != np.float32 or not r.flags.c_contiguous):
            raise TypeError("host rows must be C-contiguous float32 arrays")
    if len(rows) != channels:
        raise ValueError(f"expected {channels} channel rows, got {len(rows)}")
    arr = (ctypes.c_void_p * channels)(*[(r.__array_interface__["data"][0] if r is not None else None)
                                         for r in rows])
    return rows, arr


def _rows_device(buf, channels: int):
    """Per-channel row pointers of a device buffer (tensor with .data_ptr() and rows)."""
    if hasattr(buf, "data_ptr") and getattr(buf, "dim", lambda: 0)() == 2:
        if not buf.is_contiguous():
            raise TypeError("device buffers must be contiguous")
        stride = buf.stride(0) * buf.element_size()
        base = buf.data_ptr()
        ptrs = [base + c * stride for c in range(buf.shape[0])]
    else:
        ptrs = [(r.data_ptr() if hasattr(r, "data_ptr") else r) for r in buf]
    if len(ptrs) != channels:
        raise ValueError(f"expected {channels} channel rows, got {len(ptrs)}")
    return buf, (ctypes.c_void_p * channels)(*ptrs)


def _flags(flags, channels: int):
    if flags is None:
        return None, None
    f = np.ascontiguousarray(np.asarray(flags, dtype=np.uint32))
    if f.size != channels:
        raise ValueError("one flag mask per channel")
    return f, f.ctypes.data_as(_u32p)


class TANContext:
    """TANCreateContext (TrueAudioNext.h:647): a context bound to one CUDA device."""

    def __init__(self, device: int = 0, version: int = TAN_FULL_VERSION):
        h = ctypes.c_void_p()
        rc = lib().tanb_create_context(version, device, ctypes.byref(h))
        if rc != AMF_OK:
            raise TANError(rc, "TANCreateContext")
        self._h = h
        self.device = device

    def Release(self):
        if self._h:
            lib().tanb_context_release(self._h)
            self._h = None


class TANConvolution:
    """TANCreateConvolution + the TANConvolution interface (TrueAudioNext.h:125-253)."""

    def __init__(self, context: TANContext):
        h = ctypes.c_void_p()
        rc = lib().tanb_create_convolution(context._h, ctypes.byref(h))
        if rc != AMF_OK:
            raise TANError(rc, "TANCreateConvolution")
        self._ctx = context
        self._h = h
        self.channels = 0
        self.block = 0

    # -- lifetime -----------------------------------------------------------
    def Init(self, method: int, responseLengthInSamples: int, bufferSizeInSamples: int, channels: int) -> int:
        rc = lib().tanb_convolution_init(self._h, method, responseLengthInSamples, bufferSizeInSamples, channels)
        if rc == AMF_OK:
            self.channels, self.block = channels, bufferSizeInSamples
        return rc

    InitGpu = Init
    InitCpu = Init

    def InitNonUniform(self, method: int, responseLengthInSamples: int, bufferSizeInSamples: int, channels: int,
                       levels) -> int:
        """Init of a non-uniform method with an explicit level schedule
        [(block, partitions), ...], levels[0][0] == bufferSizeInSamples."""
        nl = len(levels)
        blocks = (ctypes.c_uint32 * nl)(*[b for b, _ in levels])
        parts = (ctypes.c_uint32 * nl)(*[k for _, k in levels])
        rc = lib().tanb_convolution_init_nu(self._h, method, responseLengthInSamples, bufferSizeInSamples, channels,
                                            nl, blocks, parts)
        if rc == AMF_OK:
            self.channels, self.block = channels, bufferSizeInSamples
        return rc

    def Terminate(self) -> int:
        return lib().tanb_convolution_terminate(self._h)

    def Release(self):
        if self._h:
            lib().tanb_convolution_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Release()
        except Exception:
            pass

    # -- IR updates ---------------------------------------------------------
    def UpdateResponseTD(self, ppBuffer, numOfSamplesToProcess: int, flagMasks=None, operationFlags: int = 0) -> int:
        keep, rows = _rows_host(ppBuffer, self.channels)
        fk, fp = _flags(flagMasks, self.channels)
        return lib().tanb_convolution_update_response_td(self._h, rows, numOfSamplesToProcess, fp, operationFlags)

    def UpdateResponseTDDevice(self, ppBuffer, numOfSamplesToProcess: int, flagMasks=None,
                               operationFlags: int = 0) -> int:
        keep, rows = _rows_device(ppBuffer, self.channels)
        fk, fp = _flags(flagMasks, self.channels)
        return lib().tanb_convolution_update_response_td_device(self._h, rows, numOfSamplesToProcess, fp,
                                                                operationFlags)

    def UpdateResponseFD(self, ppBuffer, numOfSamplesToProcess: int, flagMasks=None, operationFlags: int = 0) -> int:
        rows = (ctypes.c_void_p * max(1, self.channels))()
        return lib().tanb_convolution_update_response_fd(self._h, rows, numOfSamplesToProcess, None, operationFlags)

    # -- processing ---------------------------------------------------------
    def Process(self, ppBufferInput, ppBufferOutput, numOfSamplesToProcess: int, flagMasks=None):
        """Host buffers. Returns (AMF_RESULT, samples processed)."""
        ki, rin = _rows_host(ppBufferInput, self.channels)
        ko, rout = _rows_host(ppBufferOutput, self.channels)
        fk, fp = _flags(flagMasks, self.channels)
        done = ctypes.c_size_t(0)
        rc = lib().tanb_convolution_process(self._h, rin, rout, numOfSamplesToProcess, fp, ctypes.byref(done))
        return rc, done.value

    def ProcessHostToDevice(self, ppBufferInput, ppDeviceOutput, numOfSamplesToProcess: int, flagMasks=None):
        ki, rin = _rows_host(ppBufferInput, self.channels)
        ko, rout = _rows_device(ppDeviceOutput, self.channels)
        fk, fp = _flags(flagMasks, self.channels)
        done = ctypes.c_size_t(0)
        rc = lib().tanb_convolution_process_host_to_device(self._h, rin, rout, numOfSamplesToProcess, fp,
                                                           ctypes.byref(done))
        return rc, done.value

    def ProcessDevice(self, ppDeviceInput, ppDeviceOutput, numOfSamplesToProcess: int, flagMasks=None):
        """Device buffers; asynchronous on the object's stream (see Synchronize)."""
        ki, rin = _rows_device(ppDeviceInput, self.channels)
        ko, rout = _rows_device(ppDeviceOutput, self.channels)
        fk, fp = _flags(flagMasks, self.channels)
        done = ctypes.c_size_t(0)
        rc = lib().tanb_convolution_process_device(self._h, rin, rout, numOfSamplesToProcess, fp, ctypes.byref(done))
        return rc, done.value

    def ProcessDirect(self, ppImpulseResponse, ppBufferInput, ppBufferOutput, numOfSamplesToProcess: int,
                      nzFirstLast=None):
        kr, rir = _rows_host(ppImpulseResponse, self.channels)
        ki, rin = _rows_host(ppBufferInput, self.channels)
        ko, rout = _rows_host(ppBufferOutput, self.channels)
        nz = None
        if nzFirstLast is not None:
            nzk = np.ascontiguousarray(np.asarray(nzFirstLast, dtype=np.int32))
            nz = nzk.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        done = ctypes.c_size_t(0)
        rc = lib().tanb_convolution_process_direct(self._h, rir, rin, rout, numOfSamplesToProcess,
                                                   ctypes.byref(done), nz)
        return rc, done.value

    def ProcessMixPcm16(self, x16, in_step: int, in_gain: float, group, ngroups: int, out16, out_step: int,
                        out_gain: float, numOfSamplesToProcess: int):
        """Fused int16 -> convolution -> mix -> int16 pipeline on host rows:
        x16 (channels rows of int16, read with in_step), out16 (ngroups rows
        of int16, written with out_step). Returns (rc, clipped, done)."""
        ins = (ctypes.c_void_p * len(x16))(*[r.ctypes.data for r in x16])
        outs = (ctypes.c_void_p * len(out16))(*[r.ctypes.data for r in out16])
        g = np.ascontiguousarray(np.asarray(group, dtype=np.uint32))
        clip = ctypes.c_int32(0)
        done = ctypes.c_size_t(0)
        rc = lib().tanb_convolution_process_mix_pcm16(self._h, ins, in_step, in_gain,
                                                      g.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ngroups,
                                                      outs, out_step, out_gain, numOfSamplesToProcess,
                                                      ctypes.byref(clip), ctypes.byref(done))
        return rc, bool(clip.value), done.value

    def ProcessFinalize(self) -> int:
        return lib().tanb_convolution_process_finalize(self._h)

    def GetNextFreeChannel(self, flagMasks=None):
        idx = ctypes.c_uint32(0)
        fk, fp = _flags(flagMasks, self.channels)
        rc = lib().tanb_convolution_get_next_free_channel(self._h, ctypes.byref(idx), fp)
        return rc, idx.value

    # -- extras (no reference counterpart) ---------------------------------
    def Synchronize(self) -> int:
        return lib().tanb_convolution_synchronize(self._h)

    def stream(self) -> int:
        return lib().tanb_convolution_stream(self._h) or 0

    def tiling(self, index: int = -1):
        """Selects compiled tail tiling `index` (>= 0) and returns (AMF_RESULT, (ux, sy, depth))."""
        out = (ctypes.c_int32 * 3)()
        rc = lib().tanb_convolution_tiling(self._h, index, out)
        return rc, tuple(out)

    def Snapshot(self):
        """(AMF_RESULT, uint8 array): the object's stream state (no reference counterpart)."""
        n = ctypes.c_uint64(0)
        rc = lib().tanb_convolution_snapshot_bytes(self._h, ctypes.byref(n))
        if rc != AMF_OK:
            return rc, None
        buf = np.empty(n.value, np.uint8)
        rc = lib().tanb_convolution_snapshot(self._h, buf.ctypes.data, n.value)
        return rc, (buf if rc == AMF_OK else None)

    def Restore(self, snapshot) -> int:
        """Loads a Snapshot() of an object with the same Init into this one."""
        buf = np.ascontiguousarray(snapshot, dtype=np.uint8)
        return lib().tanb_convolution_restore(self._h, buf.ctypes.data, buf.size)

    def call_times(self) -> dict:
        """Host microseconds of the last Process call, by part."""
        us = (ctypes.c_double * 6)()
        lib().tanb_convolution_call_times(self._h, us)
        out = dict(zip(("stage_us", "launch_us", "wait_us", "copy_us", "total_us"), list(us)))
        out["in_place"] = int(us[5])  # 1: caller's input rows, 2: output rows (pinned, strided)
        return out

    def profile(self, enable: bool) -> int:
        return lib().tanb_convolution_profile(self._h, 1 if enable else 0)

    def profile_read(self) -> dict:
        """Launch counts and device ms per kernel since the last read."""
        counts = (ctypes.c_int64 * 6)()
        ms = (ctypes.c_double * 3)()
        lib().tanb_convolution_profile_read(self._h, counts, ms)
        names = ("head", "tail", "ir_spectrum")
        return {n: {"launches": counts[i], "timed": counts[3 + i], "ms": ms[i]} for i, n in enumerate(names)}

    def info(self) -> dict:
        out = (ctypes.c_int64 * 4)()
        lib().tanb_convolution_info(self._h, out)
        return {"partitions": out[0], "block": out[1], "channels": out[2], "device_bytes": out[3]}
