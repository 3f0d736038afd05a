"""The reference-side binding compiles against the reference's own headers.

tests/cpp/reference_binding.cpp holds the operators and the plan node a VelODB
maintainer adds to the reference tree (subclasses of velodb::UnaryOperator,
velodb::BinaryOperator and velodb::AbstractPlanNode that call this library's
C ABI in place of the TaskManager).  This test compiles it with g++ against
the reference's include/ directory -- with the two inputs the reference's
build system would provide: common/constants.hpp generated from its
constants.hpp.in template, and an empty stand-in for the backward-cpp header
that its exception code includes -- plus fmt header-only, and checks that
every velo_* symbol the object needs is exported by libvelo_obl.so.  It runs
where the reference tree is present and is skipped elsewhere.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("VELO_REFERENCE_TREE", "/root/reference")
SRC = os.path.join(ROOT, "tests", "cpp", "reference_binding.cpp")
LIB = os.path.join(ROOT, "velodb_b200", "libvelo_obl.so")


def _torch_include():
    import torch

    return os.path.join(os.path.dirname(torch.__file__), "include")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include", "operator")),
                    reason="the reference source tree is not on this machine")
def test_reference_binding_compiles_against_reference_headers(tmp_path):
    gen = tmp_path / "gen"
    (gen / "common").mkdir(parents=True)
    template = open(os.path.join(REF, "include", "common", "constants.hpp.in")).read()
    (gen / "common" / "constants.hpp").write_text(re.sub(r"@[A-Za-z_]+@", "0", template))
    (gen / "backward.hpp").write_text("#pragma once\n")
    obj = tmp_path / "binding.o"
    cmd = ["g++", "-std=c++20", "-c", "-o", str(obj), "-DFMT_HEADER_ONLY", "-I", os.path.join(REF, "include"),
           "-I", str(gen), "-I", os.path.join(ROOT, "include"), "-isystem", _torch_include(),
           "-I", "/usr/local/cuda/include", SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    need = {line.split()[-1] for line in subprocess.run(["nm", "-u", str(obj)], capture_output=True,
                                                        text=True).stdout.splitlines() if " velo_" in line}
    assert {"velo_submit", "velo_wait", "velo_init", "velo_ogroupby", "velo_ojoin_mn_scratch_bytes",
            "velo_ohash_join_scratch_bytes"} <= need
    if os.path.exists(LIB):
        have = {line.split()[-1] for line in subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True,
                                                            text=True).stdout.splitlines()}
        assert need <= have, sorted(need - have)
