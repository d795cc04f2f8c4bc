"""The reference-signature C++ shims (include/mertens_dr.hpp, mertens_cuda.cuh).

CPU: the reference's call pattern compiles against them and links with
libdrb200.so.  GPU: the compiled program passes the reference's known answers.
"""
import os
import subprocess

import pytest

import dr_b200
from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "shim_kat.cpp")


def _build(tmp_path):
    libdir = os.path.dirname(dr_b200.build_library())
    exe = str(tmp_path / "shim_kat")
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", libdir, "-ldrb200", f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True)
    return exe


def test_shims_compile_and_link(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_shims_known_answers(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failed" in r.stdout
