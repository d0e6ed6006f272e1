"""C++ host code drives the library through the C ABI (include/aprl_gpu.hpp):
it compiles and links on any host and runs two coupled steps on a GPU."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "host_driver.cpp")
LIBDIR = os.path.join(REPO, "aprl_b200")


def build(tmp_path):
    exe = str(tmp_path / "host_driver")
    subprocess.check_call(["g++", "-std=c++14", "-O1", "-I", os.path.join(REPO, "include"),
                           SRC, "-o", exe, "-L", LIBDIR, "-laprl_b200",
                           f"-Wl,-rpath,{LIBDIR}"])
    return exe


def test_cpp_host_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_cpp_host_runs_steps(tmp_path):
    out = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "steps=2" in out.stdout
