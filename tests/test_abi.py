"""The C ABI without a GPU: the library loads, exports every function its
header declares, lays out mb2_step_params as a C compiler does, mixes BD seeds
like the reference, and fails with a status code (never a crash) when called
without a context or without a device."""
import ctypes as C
import os
import subprocess

import pytest

from mars_md_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(lib_built):
    return _lib.load()


def test_every_header_function_is_exported(lib):
    names = _lib.header_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing
    assert lib.mb2_version() >= 100


def test_loading_a_missing_library_fails_loudly(monkeypatch):
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.load(os.path.join(ROOT, "no_such_dir", "libmarsb200.so"))


def test_step_params_layout_matches_c(tmp_path):
    fields = [f for f, _ in _lib.StepParams._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'  printf("{f} %zu\\n", offsetof(mb2_step_params, {f}));\n' for f in fields)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "marsb200.h"\n'
                   "int main(void) {\n"
                   '  printf("sizeof %zu\\n", sizeof(mb2_step_params));\n' + body + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                       text=True).stdout.splitlines())
    assert int(out["sizeof"]) == C.sizeof(_lib.StepParams)
    for f in fields:
        assert int(out[f]) == getattr(_lib.StepParams, f).offset, f


def test_bd_seed_mixing_matches_oracle(lib, oracle):
    for seed, patch, step in [(0, 0, 0), (20261203, 0, 1), (1, 2, 3), (2**64 - 1, 7, 2**40)]:
        assert lib.mb2_bd_seed(seed, patch, step) == oracle.bd_seed(seed, patch, step)


def test_null_context_is_an_argument_error(lib):
    f3 = (C.c_float * 3)(1.0, 1.0, 1.0)
    i3 = (C.c_int * 3)(1, 1, 1)
    assert lib.mb2_set_box(None, f3, f3, i3) == _lib.MB2_ERR_ARG
    assert lib.mb2_radix_sort_pairs(None, None, None, 0, None) == _lib.MB2_ERR_ARG
    assert lib.mb2_radix_sort_pairs_static(None, None, None, 0, None) == _lib.MB2_ERR_ARG
    assert lib.mb2_destroy(None) == _lib.MB2_ERR_ARG
    assert lib.mb2_last_error(None) == b"null context"


def test_create_without_a_device_reports_cuda_error(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert lib.mb2_create(0, 16, C.byref(h)) == _lib.MB2_ERR_CUDA
    assert h.value is None
