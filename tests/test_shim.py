"""The C++ drop-in header builds against unchanged reference-style caller code
(CPU), and the resulting program correlates bit-exactly on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "shim_check.cpp")
LIBDIR = os.path.join(ROOT, "ftd_b200")
CUDA = "/usr/local/cuda"


def build(out):
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", SRC, "-o", out,
           "-I", os.path.join(ROOT, "ftd_b200", "csrc", "shim"), "-I", os.path.join(ROOT, "include"),
           "-I", f"{CUDA}/include", "-L", LIBDIR, "-lftdx", f"-Wl,-rpath,{LIBDIR}",
           "-L", f"{CUDA}/lib64", "-lcudart", f"-Wl,-rpath,{CUDA}/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_shim_caller_compiles_and_links(tmp_path):
    build(str(tmp_path / "shim_check"))
    assert os.path.exists(tmp_path / "shim_check")


@pytest.mark.gpu
def test_shim_caller_runs_bit_exact(tmp_path):
    exe = str(tmp_path / "shim_check")
    build(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
