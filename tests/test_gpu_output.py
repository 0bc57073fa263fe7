"""The output side through the C ABI (mb2_output_*): DCD files byte-equal to
the reference DcdWriter's (tests/golden/dcd.npz) apart from the two title
lines (file name, date), rows in global-id order after a permutation, the
Langevin momentum DCD, restart files, the energy file and its FP64 sums."""
import os

import numpy as np
import pytest
import torch

import dcd as dcdio
from conftest import GOLDEN
from mars_md_b200 import _lib as L
from mars_md_b200 import engine as E

pytestmark = pytest.mark.gpu


def _golden():
    return np.load(os.path.join(GOLDEN, "dcd.npz"))


def _masked(buf):
    b = bytearray(buf)
    for lo, hi in dcdio.title_spans(b):
        b[lo:hi] = b" " * (hi - lo)
    return bytes(b)


@pytest.mark.parametrize("tag,cell,nf", [("cell", 1, 3), ("nocell", 0, 2)])
def test_dcd_matches_reference_writer(tmp_path, tag, cell, nf):
    d = _golden()
    n = d["frames"].shape[1]
    rng = np.random.default_rng(5)
    perm = rng.permutation(n).astype(np.int32)           # slot s holds global id perm[s]
    name = str(tmp_path / tag)
    out = E.Output(name, n, output_period=int(d["nsavc"]), timestep=float(d["delta"]),
                   box=d["box"], periodic=(cell, cell, cell))
    ids = torch.from_numpy(perm).cuda()
    for f in range(nf):
        slots = np.ascontiguousarray(d["frames"][f][perm])
        out.frame(torch.from_numpy(slots).cuda(), ids=ids)
    out.flush()
    out.close()
    got = open(name + ".dcd", "rb").read()
    ref = d[f"bytes_{tag}"].tobytes()
    assert len(got) == len(ref)
    assert _masked(got) == _masked(ref)
    r = dcdio.read_dcd(got)
    # title lines are cut or padded to 80 characters, as DcdWriter::padString does
    assert r["titles"][0] == f"REMARKS FILENAME={name}.dcd CREATED BY MARS2"[:80].ljust(80)
    assert r["titles"][1].startswith("REMARKS DATE: ")


def test_dcd_existing_file_moves_aside(tmp_path):
    name = str(tmp_path / "run")
    open(name + ".dcd", "wb").write(b"old")
    out = E.Output(name, 8)
    out.frame(torch.zeros((8, 4), dtype=torch.float32, device="cuda"))
    out.close()
    assert open(name + ".dcd.BAK", "rb").read() == b"old"
    assert dcdio.read_dcd(open(name + ".dcd", "rb").read())["nfile"] == 1


def test_momentum_output_restart_and_energy(tmp_path):
    n = 1000
    rng = np.random.default_rng(9)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-50, 50, (n, 3)).astype(np.float32)
    mom = np.zeros((n, 4), np.float32)
    mom[:, :3] = rng.normal(0, 30, (n, 3)).astype(np.float32)
    fe = np.zeros((n, 4), np.float32)
    fe[:, 3] = rng.normal(0, 2, n).astype(np.float32)
    types = rng.integers(0, 3, n).astype(np.int32)
    mass = np.array([12.0, 40.0, 100.0], np.float32)
    perm = rng.permutation(n).astype(np.int32)
    name = str(tmp_path / "lang")
    out = E.Output(name, n, output_period=5, energy_output_period=10, timestep=0.2,
                   box=(100.0, 100.0, 100.0), with_momentum=True)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v[perm])).cuda()
           for k, v in (("pos", pos), ("mom", mom), ("fe", fe), ("types", types))}
    ids = torch.from_numpy(perm).cuda()
    kT = 0.5862
    for step in (5, 10):
        out.handle_output(step, dev["pos"], dev["fe"], dev["types"], kT, mom=dev["mom"],
                          mass=mass, ids=ids)
    out.flush()
    ke, pe = out.energy(dev["fe"], kT, mom=dev["mom"], type_ids=dev["types"], mass=mass)
    out.close()
    # frames (positions and momenta) in global-id order
    r = dcdio.read_dcd(open(name + ".dcd", "rb").read())
    rm = dcdio.read_dcd(open(name + ".0.momentum.dcd", "rb").read())
    assert r["nfile"] == 2 and rm["nfile"] == 2
    assert np.array_equal(r["frames"][1], pos[:, :3]) and np.array_equal(rm["frames"][0], mom[:, :3])
    # energies: FP64 sums as write_energy_output forms them
    l2 = (mom[:, 0] * mom[:, 0] + mom[:, 1] * mom[:, 1]) + mom[:, 2] * mom[:, 2]
    ke_ref = float(np.sum(0.5 * l2.astype(np.float64) / mass[types].astype(np.float64)))
    ke_ref = ke_ref / float(np.float32(2.046167337) * np.float32(2.046167337)) / float(np.float32(kT))
    pe_ref = float(np.sum(fe[:, 3].astype(np.float64)))
    assert abs(ke - ke_ref) <= 1e-9 * abs(ke_ref) and abs(pe - pe_ref) <= 1e-9 * abs(pe_ref) + 1e-9
    lines = open(name + ".energy.dat").read().splitlines()
    assert len(lines) == 4
    assert lines[2] == "Kinetic Energy: %g (kT) " % ke and lines[3] == "Potential Energy: %g (kcal/mol) " % pe
    # restart files: "type x y z" in id order, values round-trip to float32
    for fname, arr in ((".restart", pos), (".0.momentum.restart", mom)):
        rows = [ln.split() for ln in open(name + fname).read().splitlines()]
        assert len(rows) == n
        assert [int(t[0]) for t in rows] == types.tolist()
        vals = np.array([[np.float32(x) for x in t[1:]] for t in rows], np.float32)
        assert np.array_equal(vals, arr[:, :3])
        assert max(len(x.lstrip("-").replace(".", "").split("e")[0].lstrip("0")) for t in rows
                   for x in t[1:]) <= 9


def test_bad_global_ids_are_reported(tmp_path):
    n = 64
    out = E.Output(str(tmp_path / "bad"), n)
    ids = torch.arange(n, dtype=torch.int32, device="cuda")
    ids[3] = n + 5
    out.frame(torch.zeros((n, 4), dtype=torch.float32, device="cuda"), ids=ids)
    with pytest.raises(L.MB2Error):
        out.flush()
    out.close()
