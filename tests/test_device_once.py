"""Per-device once flags of the kernel launchers (flagfft_b200/csrc/
device_once.hpp): a kernel's shared-memory limit is set per device, so the
record that it was set must be kept per device id.  Host-only: compiles and
runs a small C++ driver."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_device_once_records_per_device(tmp_path):
    cxx = shutil.which(os.environ.get("CXX", "g++")) or shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "device_once_check"
    subprocess.run([cxx, "-std=c++17", "-O1", f"-I{ROOT / 'flagfft_b200' / 'csrc'}",
                    str(ROOT / "tests" / "native" / "device_once_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "device_once ok" in out.stdout
