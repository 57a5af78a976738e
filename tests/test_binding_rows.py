"""Row arguments of the Python binding (tan_b200/convolution.py), checked on
the host before any call into the library: per-channel pointer tables from
(channels, samples) arrays or lists of rows, null rows, rejection of buffers
the kernels cannot read as rows (wrong dtype, non-contiguous, wrong channel
count), and one flag mask per channel."""
import ctypes

import numpy as np
import pytest
import torch

from tan_b200 import convolution as cv


def test_host_rows_from_a_2d_array():
    x = np.zeros((3, 256), np.float32)
    keep, arr = cv._rows_host(x, 3)
    assert len(arr) == 3
    assert [arr[c] for c in range(3)] == [x[c].ctypes.data for c in range(3)]
    assert keep[1] is not None


def test_host_rows_from_a_list_with_a_null_row():
    rows = [np.ones(64, np.float32), None, np.ones(64, np.float32)]
    _, arr = cv._rows_host(rows, 3)
    assert arr[0] == rows[0].ctypes.data and arr[1] is None and arr[2] == rows[2].ctypes.data


@pytest.mark.parametrize("bad", [np.zeros((2, 64), np.float64), np.zeros((2, 128), np.float32)[:, ::2],
                                 [np.zeros(64, np.float32), np.zeros(64, np.int16)]])
def test_host_rows_reject_what_kernels_cannot_read(bad):
    with pytest.raises(TypeError):
        cv._rows_host(bad, 2)


def test_host_rows_reject_a_wrong_channel_count():
    with pytest.raises(ValueError):
        cv._rows_host(np.zeros((3, 64), np.float32), 4)


def test_device_rows_follow_the_row_stride():
    t = torch.zeros((4, 96), dtype=torch.float32)
    _, arr = cv._rows_device(t, 4)
    assert [arr[c] for c in range(4)] == [t.data_ptr() + c * 96 * 4 for c in range(4)]
    rows = [t[c, 32:64] for c in range(4)]
    _, arr = cv._rows_device(rows, 4)
    assert [arr[c] for c in range(4)] == [t.data_ptr() + (c * 96 + 32) * 4 for c in range(4)]


def test_device_rows_reject_a_column_slice_and_a_wrong_count():
    t = torch.zeros((4, 96), dtype=torch.float32)
    with pytest.raises(TypeError):
        cv._rows_device(t[:, 32:64], 4)
    with pytest.raises(ValueError):
        cv._rows_device(t, 3)


def test_flags_one_mask_per_channel():
    assert cv._flags(None, 4) == (None, None)
    f, p = cv._flags([1, 0, 2, 3], 4)
    assert f.dtype == np.uint32 and list(f) == [1, 0, 2, 3]
    assert ctypes.cast(p, ctypes.c_void_p).value == f.ctypes.data
    with pytest.raises(ValueError):
        cv._flags([1, 2], 4)
