"""The drop-in headers compile without a GPU: include/lzk.h as C and C++,
include/lzk_compat.hpp with the reference's call shapes (tests/compat/)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
CUDA_INC = "/usr/local/cuda/include"


def _cc(args):
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "lzk.h"\nint main(void) { lzk_msm_cfg c = {0}; (void)c; return 0; }\n')
    _cc(["/usr/bin/gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", INC, str(src)])


def test_compat_driver_compiles(tmp_path):
    if not os.path.isdir(CUDA_INC):
        pytest.skip("CUDA headers not installed")
    _cc(["/usr/bin/g++", "-std=c++17", "-Wall", "-fsyntax-only", "-I", INC, "-I", CUDA_INC,
         os.path.join(ROOT, "tests", "compat", "msm_check.cpp")])


def test_groth16_class_compiles(tmp_path):
    if not os.path.isdir(CUDA_INC):
        pytest.skip("CUDA headers not installed")
    _cc(["/usr/bin/g++", "-std=c++17", "-Wall", "-fsyntax-only", "-I", INC, "-I", CUDA_INC,
         os.path.join(ROOT, "tests", "compat", "groth16_check.cpp")])
