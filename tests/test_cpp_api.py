"""The C++ API (include/fecl_b200_fec.hpp, namespace fec): a program written against
FeCl's classes compiles with g++ against the header, links libfecl_b200.so and runs
the reference's operations (tests/cpp/fec_api_test.cpp).  The host part runs on CPU;
decode and soDecode run on the GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def api_test_binary(tmp_path_factory):
    import fecl_b200
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    libdir = os.path.dirname(fecl_b200.lib_path)
    out = str(tmp_path_factory.mktemp("cpp") / "fec_api_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "fec_api_test.cpp"), "-o", out, "-L", libdir, "-lfecl_b200",
           "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def run(binary, mode):
    r = subprocess.run([binary, mode], capture_output=True, text=True, timeout=600)
    failed = [line for line in r.stdout.splitlines() if line.startswith("FAIL")]
    assert r.returncode == 0 and not failed, r.stdout[-4000:] + r.stderr[-2000:]
    return r.stdout


def test_cpp_api_host_operations(api_test_binary):
    out = run(api_test_binary, "cpu")
    assert "0 failure(s)" in out


@pytest.mark.gpu
def test_cpp_api_decode(api_test_binary):
    out = run(api_test_binary, "gpu")
    assert "lte K=6144: decode" in out and "dvbs2 16200 1/2: soDecode output sizes" in out
