"""The C++ host mirror (coral_b200/host/coral.hpp) compiles with every
wrapper called, links against libcoral_b200, and on a host without an sm_100
device every call reports CORAL_ERR_NO_DEVICE through coral::Error: the
library has no CPU fallback."""
import os
import subprocess

import pytest
import torch

from coral_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_host_mirror_reports_no_device(tmp_path):
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "host_mirror_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "coral_b200", "host"),
                    os.path.join(ROOT, "tests", "cpp", "host_mirror_test.cpp"),
                    "-L", lib_dir, "-lcoral_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "no-device", r.stdout
