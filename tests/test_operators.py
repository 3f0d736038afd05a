"""The C++ operator layer (include/velo_operator.hpp, libvelo_operators.so):
its tests are a C++ program (tests/cpp/operator_tests.cpp) built here and
linked against the operator library, the C-ABI library and the oracle."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "operator_tests.cpp")
OUT_DIR = os.path.join(ROOT, "tests", "cpp", "_build")
BIN = os.path.join(OUT_DIR, "operator_tests")
PKG = os.path.join(ROOT, "velodb_b200")
ORACLE = os.path.join(ROOT, "oracle")


@pytest.fixture(scope="module")
def operator_tests():
    from velodb_b200 import build as B

    B.build_operators()
    subprocess.run(["make", "-s", "-C", ORACLE], check=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", ORACLE, SRC,
           "-L", PKG, "-lvelo_operators", "-lvelo_obl", "-L", ORACLE, "-loracle",
           f"-Wl,-rpath,{PKG}:{ORACLE}", "-o", BIN]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return BIN


def test_operator_tests_build_and_list(operator_tests):
    r = subprocess.run([operator_tests, "--list"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    names = r.stdout.split()
    assert "order_by_mixed_directions_and_ties" in names and "hash_join_with_masks" in names


def test_operator_layer_without_device(operator_tests):
    import torch

    if torch.cuda.is_available():
        pytest.skip("covered by the GPU run")
    r = subprocess.run([operator_tests, "--no-device"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok no_device_context_error" in r.stdout and "ok schema_lookup" in r.stdout


@pytest.mark.gpu
def test_operators_on_device(cuda, operator_tests):
    r = subprocess.run([operator_tests], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failed" in r.stdout
