"""Builds and runs the C++ host-interface test program (tests/cpp) on the GPU."""
import os
import subprocess

import pytest

from gpu_util import wos

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_host_interface(tmp_path):
    import oracle as O
    O.build()
    exe = tmp_path / "host_api_test"
    libdir = os.path.dirname(wos.LIB_PATH)
    odir = os.path.join(ROOT, "oracle", "_build")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "host_api_test.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lwosgpu", "-L", odir, "-lwos_oracle",
                    f"-Wl,-rpath,{libdir}", f"-Wl,-rpath,{odir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout, r.stderr)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok")
