"""The C++ adapter (include/tanb_convolution.hpp) compiles against the C ABI
and links libtanb.so; on a GPU the compiled program passes its known answer."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_adapter.cpp")
LIBDIR = os.path.join(ROOT, "tan_b200")


def _compile(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = str(tmp_path / "test_adapter")
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-ltanb", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_adapter_compiles_and_links(tmp_path):
    assert os.path.exists(_compile(tmp_path))


@pytest.mark.gpu
def test_adapter_known_answer_on_gpu(tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
