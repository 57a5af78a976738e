"""GPU-resident room response producer (tanb_room_* of include/tanb.h): the
left / right IRs of a shoebox room written into device memory, ready for
UpdateResponseTDDevice. Mirrors the GPU path of
TrueAudioVR::generateRoomResponse (samples/src/TrueAudioVR/TrueAudioVR.cpp:659-786)."""
from __future__ import annotations

import ctypes

from . import convolution as cv
from .convolution import lib

GENROOM_LIMIT_BOUNCES = 0x40


class Room(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("width", "height", "length", "damp_left", "damp_right", "damp_top",
                                              "damp_bottom", "damp_front", "damp_back")]


class Source(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class Listener(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("head_x", "head_y", "head_z", "ear_spacing", "yaw", "pitch", "roll")] + [
        ("filter_length", ctypes.c_int32), ("low_pass", ctypes.c_float * 64), ("high_pass", ctypes.c_float * 64)]


def listener(head, ear_spacing, yaw, pitch, roll, low_pass, high_pass) -> Listener:
    L = Listener(*head, ear_spacing, yaw, pitch, roll)
    n = len(low_pass)
    L.filter_length = n
    for i in range(n):
        L.low_pass[i] = float(low_pass[i])
        L.high_pass[i] = float(high_pass[i])
    return L


class RoomGenerator:
    def __init__(self, ctx: cv.TANContext, max_length: int):
        h = ctypes.c_void_p()
        rc = lib().tanb_room_generator_create(ctx._h, max_length, ctypes.byref(h))
        if rc != cv.AMF_OK:
            raise cv.TANError(rc, "room generator")
        self._h = h.value

    def response(self, room: Room, source: Source, ears: Listener, sample_rate: int, length: int, left, right,
                 flags: int = 0, max_bounces: int = 0, stream: int = 0) -> int:
        """left / right: device buffers (data_ptr() or int) of >= length floats."""
        lp = left.data_ptr() if hasattr(left, "data_ptr") else left
        rp = right.data_ptr() if hasattr(right, "data_ptr") else right
        return lib().tanb_room_response(self._h, ctypes.byref(room), ctypes.byref(source), ctypes.byref(ears),
                                        sample_rate, length, lp, rp, flags, max_bounces, stream or None)

    def images(self) -> int:
        return lib().tanb_room_images(self._h)

    def synchronize(self) -> int:
        return lib().tanb_room_generator_synchronize(self._h)

    def stream(self) -> int:
        return lib().tanb_room_generator_stream(self._h) or 0

    def release(self) -> int:
        rc = lib().tanb_room_generator_release(self._h) if self._h else cv.AMF_OK
        self._h = None
        return rc

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self.release()
        except Exception:
            pass
