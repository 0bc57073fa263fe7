"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU.

The CPU oracle (oracle/liboracle.so) is the checker for the CUDA path; it is
built on first use (gcc, seconds).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: full-size case (seconds to minutes)")


@pytest.fixture(scope="session")
def oracle():
    pyoracle.build_oracle()
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    if not pyoracle.ref_available():
        pytest.skip("reference harness not built here (needs the reference checkout)")
    return pyoracle.RefHarness()


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib_built():
    from mars_md_b200 import build
    return build.build()


@pytest.fixture()
def ctx_factory(lib_built):
    import torch
    from mars_md_b200.engine import Context
    made = []

    def make(n):
        c = Context(max(int(n), 1))
        made.append(c)
        return c
    yield make
    torch.cuda.synchronize()
    for c in made:
        c.close()


def box_of(w):
    return pyoracle.Box.make(w.box_origin, w.box_size, w.periodic)


def tableset(w):
    return pyoracle.TableSet([(t.values, t.start, t.step_inv) for t in w.pair_tables])


def u32(t):
    """torch int32 tensor -> numpy uint32 (bit-identical)."""
    return t.cpu().numpy().view(np.uint32)


def force_errors(f_gpu, f64_ref, fabs_sum, eps_rel=1e-5):
    """Per-particle force error relative to the sum of |pair force| magnitudes
    acting on that particle (the scale any float summation order is accurate
    to), and the plain norm-relative error. Returns (worst scaled, worst plain)."""
    d = np.linalg.norm(f_gpu[:, :3].astype(np.float64) - f64_ref[:, :3], axis=1)
    mag = np.linalg.norm(f64_ref[:, :3], axis=1)
    scale = np.maximum(fabs_sum, 1e-30)
    rel_scaled = np.where(fabs_sum > 0, d / scale, d)
    frms = np.sqrt(np.mean(mag ** 2)) if len(mag) else 1.0
    rel_plain = d / np.maximum(mag, 1e-3 * frms)
    return float(rel_scaled.max(initial=0.0)), float(rel_plain.max(initial=0.0))
