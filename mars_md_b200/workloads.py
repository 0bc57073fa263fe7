"""Seeded synthetic workloads for the Brownian-dynamics step.

No public dataset is involved: every input is generated here from
``numpy.random.default_rng(seed)`` (default seed 20261203) with the shapes, sizes
and value distributions of the five benchmark configurations:

* ``plain_bd``        4,096 point particles, one type, 200 A periodic cube,
                      WCA-like table (200 bins of 0.1 A), cutoff 20 A, list 25 A.
* ``polymers``        64 chains x 1,024 beads, 2 types, 600 A box, tabulated
                      harmonic bonds/angles, 1-2/1-3 exclusions, 3 pair tables,
                      256^3 cylindrical-pore grid potential.
* ``large_plain``     2,097,152 beads, 4 types, 10 pair tables of 400 bins
                      (Debye-Hueckel + soft core), cutoff 30 A, list 35 A,
                      rebuilt every 20 steps.
* ``batched``         512 replicas, sizes log-uniform in [500, 20000].
* ``adjoint``         16 chains x 1,024 beads, one type, no grid.

Physical constants follow the reference: kT = T * 0.001987191 kcal/mol
(src/Constants.h:25, src/SimParam.h:32-35); time step in ns.

Tables are described as the reference reads them from "x y" text files
(src/Objects/Tables.h:27-120): X and Y are float32; step = X[1] - X[0] in
float; angle tables are in degrees and converted to radians in float. The
non-bonded step inverse is ``1.0f / step`` (DevicePairNonBondedInteraction.h:183)
and the bonded one ``float(1.0 / double(step))`` (DeviceBondedInteraction.h:213).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

DEFAULT_SEED = 20261203
KCAL_PER_K = 0.001987191           # src/Constants.h:25
TEMPERATURE = 295.0                # K
DIFFUSION = 150.0                  # A^2/ns
DT_NS = 1e-4                       # 100 fs
DEG_TO_RAD = np.float32(math.pi / 180.0)


def kT(temperature: float = TEMPERATURE) -> float:
    return float(np.float32(np.float32(temperature) * np.float32(KCAL_PER_K)))


@dataclass
class TableSpec:
    """One tabulated potential as the reference holds it after loading."""
    values: np.ndarray        # float32 Y
    start: float              # float32 X[0] (radians for angle tables)
    step: float               # float32 X[1]-X[0] (radians for angle tables)
    periodic: bool = False
    kind: str = "pair"        # "pair" | "bond" | "angle"

    @property
    def step_inv(self) -> float:
        if self.kind == "pair":
            return float(np.float32(1.0) / np.float32(self.step))
        return float(np.float32(1.0 / float(np.float64(np.float32(self.step)))))


def table_from_xy(x: np.ndarray, y: np.ndarray, kind: str) -> TableSpec:
    """Reference loading rules: float X/Y, step = X1 - X0, degrees -> radians."""
    x = np.asarray(x, np.float32)
    y = np.asarray(y, np.float32)
    step = np.float32(x[1] - x[0])
    start = np.float32(x[0])
    if kind == "angle":
        step = np.float32(step * DEG_TO_RAD)
        start = np.float32(start * DEG_TO_RAD)
    return TableSpec(values=y, start=float(start), step=float(step),
                     periodic=(kind == "angle"), kind=kind)


def wca_table(sigma=4.0, eps=0.5, cap=20.0, bins=200, dx=0.1) -> TableSpec:
    """WCA-like pair table U = 4 eps[(s/r)^12 - (s/r)^6] + eps below 2^(1/6) s,
    0 beyond, capped at `cap` kcal/mol (finite at r = 0)."""
    x = (np.arange(bins, dtype=np.float64) * dx)
    rc = 2.0 ** (1.0 / 6.0) * sigma
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        sr6 = (sigma / x) ** 6
        u = 4.0 * eps * (sr6 * sr6 - sr6) + eps
    u = np.where(x < rc, u, 0.0)
    u = np.where(np.isfinite(u), np.minimum(u, cap), cap)
    return table_from_xy(x.astype(np.float32), u.astype(np.float32), "pair")


def dh_softcore_table(qi, qj, bins=400, rmax=30.0, r_floor=1.0) -> TableSpec:
    """Debye-Hueckel (332.0636 qi qj / (80 r) exp(-r / 10 A)) plus a soft core
    10 (1 - r / 6 A)^2 below 6 A; the Coulomb part is evaluated at max(r, 1 A)
    so the table stays finite at r = 0."""
    dx = rmax / bins
    x = np.arange(bins, dtype=np.float64) * dx
    r = np.maximum(x, r_floor)
    u = 332.0636 * qi * qj / (80.0 * r) * np.exp(-r / 10.0)
    u += np.where(x < 6.0, 10.0 * (1.0 - x / 6.0) ** 2, 0.0)
    return table_from_xy(x.astype(np.float32), u.astype(np.float32), "pair")


def harmonic_bond_table(k=10.0, r0=5.0, bins=200, dx=0.1) -> TableSpec:
    x = np.arange(bins, dtype=np.float64) * dx
    return table_from_xy(x.astype(np.float32), (0.5 * k * (x - r0) ** 2).astype(np.float32), "bond")


def harmonic_angle_table(k=5.0, theta0_deg=180.0, rows=181) -> TableSpec:
    xdeg = np.arange(rows, dtype=np.float64)
    th = np.deg2rad(xdeg)
    u = 0.5 * k * (th - math.radians(theta0_deg)) ** 2
    return table_from_xy(xdeg.astype(np.float32), u.astype(np.float32), "angle")


@dataclass
class Workload:
    name: str
    pos: np.ndarray                   # float32 [N, 4], w = 0
    type_ids: np.ndarray              # int32 [N]
    box_origin: tuple
    box_size: tuple
    periodic: tuple
    pair_tables: list                 # [TableSpec]
    term_matrix: np.ndarray           # uint32 [T*T] pair tags (bit 5 | table << 8)
    num_types: int
    cutoff: float
    list_radius: float
    rebuild_period: int
    dt: float = DT_NS
    temperature: float = TEMPERATURE
    diffusion: np.ndarray = None      # float32 [T, 3]
    charge: np.ndarray = None         # float32 [T]
    bonds: np.ndarray = None          # int32 [B, 2]
    bond_table_idx: np.ndarray = None
    bond_tables: list = field(default_factory=list)
    angles: np.ndarray = None         # int32 [A, 4] (i, j, k, 0)
    angle_table_idx: np.ndarray = None
    angle_tables: list = field(default_factory=list)
    exclusions: np.ndarray = None     # int32 [E, 2]
    grids: list = field(default_factory=list)   # dicts: data, origin, basis, boundary_condition
    pmf_terms: list = None            # per type: [(grid_id, scale, slope, bc)]
    steps: int = 1000
    seed: int = DEFAULT_SEED

    @property
    def n(self) -> int:
        return len(self.pos)

    @property
    def kT(self) -> float:
        return kT(self.temperature)


def _pair_tag(table_index: int) -> int:
    # make_pair_tag(PAIR_TERM_TABULATED, idx) (src/Interactions/Nonbonded/Pairwise.h:31-35)
    return (1 << 5) | (table_index << 8)


def _term_matrix(num_types: int, table_of_pair) -> np.ndarray:
    m = np.zeros(num_types * num_types, np.uint32)
    for a in range(num_types):
        for b in range(num_types):
            m[a * num_types + b] = _pair_tag(table_of_pair(min(a, b), max(a, b)))
    return m


def _pos4(xyz: np.ndarray) -> np.ndarray:
    p = np.zeros((len(xyz), 4), np.float32)
    p[:, :3] = xyz.astype(np.float32)
    return p


def plain_bd(seed: int = DEFAULT_SEED, n: int = 4096, box: float = 200.0) -> Workload:
    rng = np.random.default_rng(seed)
    pos = _pos4(rng.uniform(0.0, box, size=(n, 3)))
    return Workload(
        name="plain_bd", pos=pos, type_ids=np.zeros(n, np.int32), box_origin=(0.0, 0.0, 0.0),
        box_size=(box, box, box), periodic=(1, 1, 1), pair_tables=[wca_table()],
        term_matrix=_term_matrix(1, lambda a, b: 0), num_types=1, cutoff=20.0,
        list_radius=25.0, rebuild_period=20,
        diffusion=np.full((1, 3), DIFFUSION, np.float32), charge=np.zeros(1, np.float32),
        steps=1000, seed=seed)


def cylinder_pore_grid(box: float = 600.0, n: int = 256, radius=30.0, height=5.0, width=2.0):
    """256^3 grid at 1 A spacing centred in the box: U = height * smoothstep((rho - radius)
    / width), rho the distance from the grid's z axis; 0 inside the pore."""
    origin = box * 0.5 - n * 0.5
    c = np.arange(n, dtype=np.float64) + origin
    gx, gy = np.meshgrid(c, c, indexing="ij")
    rho = np.sqrt((gx - box * 0.5) ** 2 + (gy - box * 0.5) ** 2)
    t = np.clip((rho - radius) / width, 0.0, 1.0)
    plane = (height * t * t * (3.0 - 2.0 * t)).astype(np.float32)
    data = np.broadcast_to(plane[:, :, None], (n, n, n)).copy()  # index [x, y, z]
    return dict(data=data, origin=(origin, origin, origin), basis=np.eye(3, dtype=np.float32),
                boundary_condition=0)


def _chains(rng, n_chains, beads, box, bond=5.0):
    starts = rng.uniform(0.0, box, size=(n_chains, 3))
    dirs = rng.normal(size=(n_chains, beads - 1, 3))
    dirs /= np.linalg.norm(dirs, axis=2, keepdims=True)
    steps = np.concatenate([np.zeros((n_chains, 1, 3)), np.cumsum(bond * dirs, axis=1)], axis=1)
    xyz = (starts[:, None, :] + steps).reshape(-1, 3)
    return np.mod(xyz, box)


def _topology(n_chains, beads):
    idx = np.arange(n_chains * beads).reshape(n_chains, beads)
    bonds = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], axis=1).astype(np.int32)
    ang = np.stack([idx[:, :-2].ravel(), idx[:, 1:-1].ravel(), idx[:, 2:].ravel(),
                    np.zeros(n_chains * (beads - 2), np.int64)], axis=1).astype(np.int32)
    ex13 = np.stack([idx[:, :-2].ravel(), idx[:, 2:].ravel()], axis=1).astype(np.int32)
    excl = np.concatenate([bonds, ex13]).astype(np.int32)
    return bonds, ang, excl


def polymers(seed: int = DEFAULT_SEED, n_chains=64, beads=1024, box=600.0,
             with_grid=True) -> Workload:
    rng = np.random.default_rng(seed)
    xyz = _chains(rng, n_chains, beads, box)
    n = n_chains * beads
    types = np.tile((np.arange(beads) >= beads // 2).astype(np.int32), n_chains)
    bonds, angles, excl = _topology(n_chains, beads)
    tabs = [wca_table(), wca_table(sigma=4.5), wca_table(sigma=5.0)]   # AA, AB, BB
    grids = [cylinder_pore_grid(box)] if with_grid else []
    pmf = [[(0, 1.0, 0.0, -1)], [(0, 1.0, 0.0, -1)]] if with_grid else None
    return Workload(
        name="polymers", pos=_pos4(xyz), type_ids=types, box_origin=(0.0, 0.0, 0.0),
        box_size=(box, box, box), periodic=(1, 1, 1), pair_tables=tabs,
        term_matrix=_term_matrix(2, lambda a, b: a + b), num_types=2, cutoff=20.0,
        list_radius=25.0, rebuild_period=20,
        diffusion=np.full((2, 3), DIFFUSION, np.float32), charge=np.zeros(2, np.float32),
        bonds=bonds, bond_table_idx=np.zeros(len(bonds), np.int32),
        bond_tables=[harmonic_bond_table()], angles=angles,
        angle_table_idx=np.zeros(len(angles), np.int32), angle_tables=[harmonic_angle_table()],
        exclusions=excl, grids=grids, pmf_terms=pmf, steps=1000, seed=seed)


LARGE_N = 2_097_152


def large_plain(seed: int = DEFAULT_SEED, n: int = LARGE_N, density: float = 0.002) -> Workload:
    rng = np.random.default_rng(seed)
    box = float((n / density) ** (1.0 / 3.0))
    pos = _pos4(rng.uniform(0.0, box, size=(n, 3)))
    types = (np.arange(n) % 4).astype(np.int32)
    charges = [1.0, -1.0, 1.0, -1.0]
    pairs = [(a, b) for a in range(4) for b in range(a, 4)]
    tabs = [dh_softcore_table(charges[a], charges[b]) for a, b in pairs]
    index = {p: k for k, p in enumerate(pairs)}
    return Workload(
        name="large_plain", pos=pos, type_ids=types, box_origin=(0.0, 0.0, 0.0),
        box_size=(box, box, box), periodic=(1, 1, 1), pair_tables=tabs,
        term_matrix=_term_matrix(4, lambda a, b: index[(a, b)]), num_types=4, cutoff=30.0,
        list_radius=35.0, rebuild_period=20,
        diffusion=np.full((4, 3), DIFFUSION, np.float32), charge=np.zeros(4, np.float32),
        steps=10000, seed=seed)


def batched(seed: int = DEFAULT_SEED, systems=512, nmin=500, nmax=20000, density=0.002):
    """Independent replicas with log-uniform sizes; each its own periodic box at the
    given density with the plain_bd tables and cutoffs."""
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=systems))).astype(int)
    out = []
    for s, n in enumerate(sizes):
        box = float((n / density) ** (1.0 / 3.0))
        w = plain_bd(seed=seed + 1 + s, n=int(n), box=box)
        w.name = f"replica{s}"
        out.append(w)
    return out


def adjoint(seed: int = DEFAULT_SEED, n_chains=16, beads=1024) -> Workload:
    box = 600.0 * (n_chains / 64.0) ** (1.0 / 3.0)
    w = polymers(seed=seed, n_chains=n_chains, beads=beads, box=box, with_grid=False)
    w.name = "adjoint"
    w.type_ids = np.zeros(w.n, np.int32)
    w.pair_tables = [wca_table()]
    w.term_matrix = _term_matrix(1, lambda a, b: 0)
    w.num_types = 1
    w.diffusion = np.full((1, 3), DIFFUSION, np.float32)
    w.charge = np.zeros(1, np.float32)
    w.steps = 200
    return w


CONFIGS = {"plain_bd": plain_bd, "polymers": polymers, "large_plain": large_plain,
           "adjoint": adjoint}
