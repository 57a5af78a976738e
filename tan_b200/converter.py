"""Python mirror of TANConverter and TANMixer (TrueAudioNext.h:344-398,
611-634) over the C ABI of include/tanb.h. Host arrays follow the reference's
CPU results bit for bit (ConverterImpl.cpp, MixerImpl.cpp); device tensors
(anything with data_ptr()) those of its OpenCL kernels (Converter.cl,
Mixer.cl)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import convolution as cv
from .convolution import lib

TAN_SAMPLE_TYPE_FLOAT = 0
TAN_SAMPLE_TYPE_SHORT = 1


def _ptr(a) -> int:
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


class TANConverter:
    """TANCreateConverter + Init (TrueAudioNext.h:653-656, 349)."""

    def __init__(self, ctx: cv.TANContext):
        h = ctypes.c_void_p()
        rc = lib().tanb_converter_create(ctx._h, ctypes.byref(h))
        if rc != cv.AMF_OK:
            raise cv.TANError(rc, "TANCreateConverter")
        self._h = h.value

    def Terminate(self) -> int:
        rc = lib().tanb_converter_release(self._h) if self._h else cv.AMF_OK
        self._h = None
        return rc

    def ConvertShortToFloat(self, x: np.ndarray, in_step: int, n: int, y: np.ndarray, out_step: int,
                            gain: float) -> int:
        """Convert(short*, inputStep, n, float*, outputStep, gain) on host arrays."""
        return lib().tanb_converter_short_to_float(self._h, x.ctypes.data, in_step, n, y.ctypes.data, out_step, gain)

    def ConvertFloatToShort(self, x: np.ndarray, in_step: int, n: int, y: np.ndarray, out_step: int,
                            gain: float):
        """Convert(float*, ..., short*, ..., gain, &clipped) on host arrays; returns (rc, clipped)."""
        clip = ctypes.c_int32(0)
        rc = lib().tanb_converter_float_to_short(self._h, x.ctypes.data, in_step, n, y.ctypes.data, out_step, gain,
                                                 ctypes.byref(clip))
        return rc, bool(clip.value)

    def ConvertShortToFloatBatch(self, xs, in_step: int, n: int, ys, out_step: int, gain: float) -> int:
        pin = (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
        pout = (ctypes.c_void_p * len(ys))(*[y.ctypes.data for y in ys])
        return lib().tanb_converter_short_to_float_batch(self._h, pin, in_step, n, pout, out_step, gain, len(xs))

    def ConvertFloatToShortBatch(self, xs, in_step: int, n: int, ys, out_step: int, gain: float):
        pin = (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
        pout = (ctypes.c_void_p * len(ys))(*[y.ctypes.data for y in ys])
        clip = ctypes.c_int32(0)
        rc = lib().tanb_converter_float_to_short_batch(self._h, pin, in_step, n, pout, out_step, gain, len(xs),
                                                       ctypes.byref(clip))
        return rc, bool(clip.value)

    def ConvertDevice(self, xs, in_step: int, in_offsets, in_type: int, ys, out_step: int, out_offsets,
                      out_type: int, n: int, gain: float, want_clipped: bool = False):
        """Convert(cl_mem* ...) equivalent on device buffers; returns (rc, clipped or None)."""
        count = len(xs)
        pin = (ctypes.c_void_p * count)(*[_ptr(x) for x in xs])
        pout = (ctypes.c_void_p * count)(*[_ptr(y) for y in ys])
        oin = (ctypes.c_size_t * count)(*(in_offsets or [0] * count))
        oout = (ctypes.c_size_t * count)(*(out_offsets or [0] * count))
        clip = ctypes.c_int32(0)
        rc = lib().tanb_converter_convert_device(self._h, pin, in_step, oin, in_type, pout, out_step, oout, out_type,
                                                 n, gain, count, ctypes.byref(clip) if want_clipped else None)
        return rc, (bool(clip.value) if want_clipped else None)

    def Synchronize(self) -> int:
        return lib().tanb_converter_synchronize(self._h)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self.Terminate()
        except Exception:
            pass


class TANMixer:
    """TANCreateMixer + Init(buffer_size, num_channels) (TrueAudioNext.h:657-660, 616)."""

    def __init__(self, ctx: cv.TANContext, buffer_size: int, channels: int):
        h = ctypes.c_void_p()
        rc = lib().tanb_mixer_create(ctx._h, buffer_size, channels, ctypes.byref(h))
        if rc != cv.AMF_OK:
            raise cv.TANError(rc, "TANMixer.Init")
        self._h = h.value
        self.buffer_size, self.channels = buffer_size, channels

    def Terminate(self) -> int:
        rc = lib().tanb_mixer_release(self._h) if self._h else cv.AMF_OK
        self._h = None
        return rc

    def Mix(self, xs, y: np.ndarray) -> int:
        """Mix(float* in[], float* out) on host arrays."""
        pin = (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
        return lib().tanb_mixer_mix(self._h, pin, y.ctypes.data)

    def MixDevice(self, xs, y) -> int:
        """Mix(cl_mem in[], cl_mem out) on device buffers (asynchronous)."""
        pin = (ctypes.c_void_p * len(xs))(*[_ptr(x) for x in xs])
        return lib().tanb_mixer_mix_device(self._h, pin, _ptr(y))

    def MixDeviceStrided(self, x, y, input_stride: int) -> int:
        """Mix(cl_mem in, cl_mem out, inputStride) (asynchronous)."""
        return lib().tanb_mixer_mix_device_strided(self._h, _ptr(x), _ptr(y), input_stride)

    def Synchronize(self) -> int:
        return lib().tanb_mixer_synchronize(self._h)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self.Terminate()
        except Exception:
            pass
