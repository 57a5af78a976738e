"""B200-native TrueAudio Next convolution path.

libtanb.so (built from tan_b200/csrc by tan_b200.build) exposes the C ABI of
include/tanb.h; tan_b200.convolution mirrors amf::TANConvolution on top of it.
"""
from .convolution import (  # noqa: F401
    TANContext,
    TANConvolution,
    TANError,
    lib,
)
from . import convolution  # noqa: F401
