"""The C++ host mirror of the reference's Pairlist / Patch interface
(mars_md_b200/host/b200_pairlist.hpp), exercised by a C++ program written like
the reference's own pairlist tests (tests/cpp/pairlist_mirror_test.cpp)."""
import os
import subprocess

import pytest


@pytest.fixture(scope="module")
def mirror_bin(lib_built):
    from mars_md_b200.build import build_cpp_mirror_test
    return build_cpp_mirror_test()


def test_mirror_compiles_and_links(mirror_bin):
    assert os.access(mirror_bin, os.X_OK)


@pytest.mark.gpu
def test_mirror_program_passes(mirror_bin):
    r = subprocess.run([mirror_bin], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASS" in r.stdout
    assert r.stdout.count("PASS ") >= 15
