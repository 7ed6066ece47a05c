"""The C++ API (include/bmmpy/, the reference's class names over the C ABI):
tests/cpp/test_bmmpy_api.cpp is compiled with g++ against the in-tree
libbmm_b200.so and run -- host mode without a GPU (layout, argument checks,
exception types), device mode on the GPU (searches against each other, the
launch seams, known answers)."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "bmmpy_b200")


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ is not available")
    out = str(tmp_path_factory.mktemp("cpp") / "test_bmmpy_api")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "test_bmmpy_api.cpp"), "-o", out,
                    "-L", LIBDIR, "-lbmm_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return out


def test_cpp_api_host(binary):
    r = subprocess.run([binary, "host"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


@pytest.mark.gpu
def test_cpp_api_device(binary):
    r = subprocess.run([binary, "device"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"
