"""The drop-in boundary against the reference's own interface: the adapter
mars_md_b200/host/b200_ref_adapter.hpp derives from the reference's
MARS::Pairlist (src/PatchOperation/Pairlist.h:56-172), compiled against the
reference's headers, and forwards every override to the C ABI.

CPU: the adapter and its driver compile against the reference checkout (when
present here). GPU: a pairlist built through MARS::Pairlist's virtuals
(set_periodic_box, set_exclusions, build_pairlist, get_num_pairs,
get_neighbor_pairs, needs_update) holds exactly the oracle's pair set, on the
4,096-bead plain workload and on polymers with 1-2/1-3 exclusions.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import box_of
from mars_md_b200 import build as B
from mars_md_b200 import workloads as W


@pytest.fixture(scope="module")
def adapter_bin(lib_built):
    path = B.build_ref_adapter_test()
    if path is None:
        pytest.skip("no reference checkout here and no adapter test built earlier")
    return path


def test_adapter_compiles_against_reference_headers(adapter_bin):
    assert os.access(adapter_bin, os.X_OK)


def _write_case(path, w, rc, excl=None):
    with open(path, "wb") as f:
        f.write(struct.pack("<I", w.n))
        f.write(np.asarray(w.box_origin, np.float32).tobytes())
        f.write(np.asarray(w.box_size, np.float32).tobytes())
        f.write(np.asarray(w.periodic, np.int32).tobytes())
        f.write(struct.pack("<f", rc))
        f.write(struct.pack("<I", 0 if excl is None else len(excl[0])))
        f.write(np.ascontiguousarray(w.pos, np.float32).tobytes())
        if excl is not None:
            f.write(np.ascontiguousarray(excl[0], np.int32).tobytes())
            f.write(struct.pack("<I", len(excl[1])))
            f.write(np.ascontiguousarray(excl[1], np.int32).tobytes())


def _read_pairs(path):
    with open(path, "rb") as f:
        n = struct.unpack("<Q", f.read(8))[0]
        p = np.frombuffer(f.read(8 * n), np.int32).reshape(n, 2).astype(np.int64)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["plain", "polymers"])
def test_pairlist_through_reference_interface(adapter_bin, oracle, tmp_path, case):
    if case == "plain":
        w, excl, excl_np = W.plain_bd(), None, None
    else:
        w = W.polymers(n_chains=8, beads=1024, with_grid=False)
        off, nb, npart = oracle.exclusion_csr(w.exclusions)
        off = off[:w.n + 1] if len(off) >= w.n + 1 else np.pad(off, (0, w.n + 1 - len(off)),
                                                                  mode="edge")
        excl, excl_np = (off, nb[:off[-1]]), (off, nb, npart)
    src, dst = tmp_path / "case.bin", tmp_path / "pairs.bin"
    _write_case(src, w, w.list_radius, excl)
    r = subprocess.run([adapter_bin, str(src), str(dst)], capture_output=True, text=True,
                       timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASS" in r.stdout
    got = _read_pairs(dst)
    ref, cnt, _ = oracle.build_pairlist(w.pos, box_of(w), w.list_radius, excl=excl_np)
    assert len(got) == cnt
    assert np.array_equal(got, ref.astype(np.int64))
