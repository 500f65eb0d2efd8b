"""Seeded synthetic molecular systems and CHARMM file writers.

The benchmark workloads of this package are synthetic: TIP3P water boxes and a
solvated self-avoiding bead chain.  This module builds them as plain numpy
arrays (a :class:`System`) and writes them as CHARMM PSF (XPLOR format), CARD
coordinate and parameter files, which is the only input path the reference
engine accepts (``CharmmPSF::readCharmmPSF`` src/CharmmPSF.cu:387,
``CharmmParameters`` src/CharmmParameters.cu, ``CharmmCrd`` src/CharmmCrd.cu).

Conventions follow the reference:
  * the box is centred on the origin (image centering wraps a molecule when its
    centroid leaves [-L/2, L/2), src/CharmmContext.cu:276-372);
  * LJ well depths are written negative (CHARMM convention); the pair
    parameters are eps_ij = sqrt(eps_i eps_j), rmin_ij = rmin/2_i + rmin/2_j
    (src/CharmmParameters.cu:739-777);
  * TIP3P atoms are typed OT/HT so that SETTLE and the degree-of-freedom count
    engage (src/CharmmPSF.cu:281-296, src/ForceManager.cu:863).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Sequence, Tuple

import numpy as np

# TIP3P geometry and parameters (values as in the reference's
# test/data/toppar_water_ions.str:240-242 and the TIP3P paper)
R_OH = 0.9572
THETA_HOH = 104.52
Q_O, Q_H = -0.834, 0.417
M_O, M_H = 15.9994, 1.008
LJ_OT = (-0.1521, 1.7682)
LJ_HT = (-0.046, 0.2245)


@dataclasses.dataclass
class System:
    """One molecular system as flat arrays (0-based atom indices)."""

    name: str
    box: Tuple[float, float, float]
    pos: np.ndarray                 # (N,3) float64, molecules whole
    charge: np.ndarray              # (N,) float64
    mass: np.ndarray                # (N,) float64
    atom_type: List[str]            # CHARMM atom type per atom
    atom_name: List[str]
    res_name: List[str]
    res_id: List[int]
    seg_id: List[str]
    bonds: np.ndarray               # (nb,2) int
    angles: np.ndarray              # (na,3) int
    dihedrals: np.ndarray           # (nd,4) int
    impropers: np.ndarray           # (ni,4) int
    # parameters keyed by CHARMM atom types
    masses_by_type: Dict[str, float]
    bond_params: Dict[Tuple[str, str], Tuple[float, float]]          # (kb, b0)
    angle_params: Dict[Tuple[str, str, str], Tuple[float, float]]    # (ktheta, theta0 deg)
    dihedral_params: Dict[Tuple[str, str, str, str], List[Tuple[float, int, float]]]  # [(kchi, n, delta deg)]
    improper_params: Dict[Tuple[str, str, str, str], Tuple[float, float]]  # (kpsi, psi0 deg)
    lj_params: Dict[str, Tuple[float, float]]                        # (eps<0, rmin/2)
    lj14_params: Dict[str, Tuple[float, float]]
    # PME / cutoff settings the workload is quoted with
    settings: Dict[str, float] = dataclasses.field(default_factory=dict)

    @property
    def n_atoms(self) -> int:
        return int(self.pos.shape[0])


# --------------------------------------------------------------------------
# geometry helpers
# --------------------------------------------------------------------------

def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from unit quaternions (Shoemake)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([
        np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
        np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
        np.sqrt(u1) * np.sin(2 * np.pi * u3),
        np.sqrt(u1) * np.cos(2 * np.pi * u3),
    ], axis=1)
    x, y, z, w = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _water_template() -> np.ndarray:
    """O, H1, H2 in a frame with the centre of mass at the origin."""
    half = math.radians(THETA_HOH) / 2
    o = np.array([0.0, 0.0, 0.0])
    h1 = np.array([R_OH * math.sin(half), 0.0, R_OH * math.cos(half)])
    h2 = np.array([-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)])
    t = np.stack([o, h1, h2])
    com = (M_O * o + M_H * h1 + M_H * h2) / (M_O + 2 * M_H)
    return t - com


def _lattice_sites(L: float, n_per_edge: int) -> np.ndarray:
    g = (np.arange(n_per_edge) + 0.5) * (L / n_per_edge) - L / 2
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def _place_waters(rng, centres: np.ndarray, jitter: float, L: float,
                  others: np.ndarray | None = None, d_min: float = 1.5,
                  max_rounds: int = 40) -> np.ndarray:
    """Waters at jittered lattice centres with random orientations; the
    orientation (and later the jitter) of any molecule with an atom closer
    than d_min to an atom of another molecule (or of `others`) is redrawn,
    for at most max_rounds rounds.  Contacts that remain in very dense
    systems are removed by `relax` (api.py) before dynamics."""
    from scipy.spatial import cKDTree

    n = centres.shape[0]
    jit = rng.normal(0.0, jitter, size=centres.shape)
    R = _random_rotations(rng, n)
    t = _water_template()
    nother = 0 if others is None else others.shape[0]
    for rnd in range(max_rounds):
        c = centres + jit
        pos = (c[:, None, :] + np.einsum("nij,aj->nai", R, t)).reshape(-1, 3)
        allp = pos if others is None else np.concatenate([pos, others])
        tree = cKDTree(np.mod(allp + L / 2, L) % L, boxsize=L)
        pairs = tree.query_pairs(d_min, output_type="ndarray")
        mol = np.where(np.arange(len(allp)) < 3 * n, np.arange(len(allp)) // 3, -1)
        a, b = mol[pairs[:, 0]], mol[pairs[:, 1]]
        bad = a != b
        hit = np.unique(np.concatenate([a[bad & (a >= 0)], b[bad & (b >= 0)]]))
        if hit.size == 0 or rnd == max_rounds - 1:
            return pos
        R[hit] = _random_rotations(rng, hit.size)
        if rnd >= 10 and rnd % 2:
            jit[hit] = rng.normal(0.0, jitter, size=(hit.size, 3))
    return pos


# --------------------------------------------------------------------------
# systems
# --------------------------------------------------------------------------

def _water_topology(n_water: int, first_atom: int = 0, seg: str = "WAT",
                    first_res: int = 1):
    idx = first_atom + 3 * np.arange(n_water)
    bonds = np.concatenate([
        np.stack([idx, idx + 1], 1), np.stack([idx, idx + 2], 1),
        np.stack([idx + 1, idx + 2], 1)])
    # keep the reference's per-molecule order O-H1, O-H2, H1-H2
    bonds = bonds.reshape(3, n_water, 2).transpose(1, 0, 2).reshape(-1, 2)
    angles = np.stack([idx + 1, idx, idx + 2], 1)
    types, names, resn, resi, segs = [], [], [], [], []
    for m in range(n_water):
        types += ["OT", "HT", "HT"]
        names += ["OH2", "H1", "H2"]
        resn += ["TIP3"] * 3
        resi += [first_res + m] * 3
        segs += [seg] * 3
    return bonds, angles, types, names, resn, resi, segs


def _water_params():
    return dict(
        masses_by_type={"OT": M_O, "HT": M_H},
        bond_params={("HT", "HT"): (0.0, 1.5139), ("HT", "OT"): (450.0, R_OH)},
        angle_params={("HT", "OT", "HT"): (55.0, THETA_HOH)},
        lj={"OT": LJ_OT, "HT": LJ_HT},
    )


def water_box(n_molecules: int, L: float, seed: int = 2024,
              jitter: float = 0.3, name: str = "waterbox") -> System:
    """Cubic TIP3P box: molecules on a jittered lattice, random orientations."""
    rng = np.random.default_rng(seed)
    n_edge = int(math.ceil(n_molecules ** (1.0 / 3.0)))
    sites = _lattice_sites(L, n_edge)
    if sites.shape[0] > n_molecules:
        keep = np.sort(rng.choice(sites.shape[0], n_molecules, replace=False))
        sites = sites[keep]
    pos = _place_waters(rng, sites, jitter, L)
    bonds, angles, types, names, resn, resi, segs = _water_topology(n_molecules)
    p = _water_params()
    n = 3 * n_molecules
    return System(
        name=name, box=(L, L, L), pos=pos,
        charge=np.tile([Q_O, Q_H, Q_H], n_molecules).astype(np.float64),
        mass=np.tile([M_O, M_H, M_H], n_molecules).astype(np.float64),
        atom_type=types, atom_name=names, res_name=resn, res_id=resi, seg_id=segs,
        bonds=bonds.astype(np.int64), angles=angles.astype(np.int64),
        dihedrals=np.zeros((0, 4), np.int64), impropers=np.zeros((0, 4), np.int64),
        masses_by_type=p["masses_by_type"], bond_params=p["bond_params"],
        angle_params=p["angle_params"], dihedral_params={}, improper_params={},
        lj_params=p["lj"], lj14_params={},
    )


def _self_avoiding_chain(rng, n_beads: int, L: float, bond: float = 1.53,
                         theta0: float = 111.0, min_dist: float = 2.6,
                         margin: float = 1.5) -> np.ndarray:
    """Confined self-avoiding walk with fixed bond length and angle.

    Beads stay inside [-L/2+margin, L/2-margin]^3 so the molecule never crosses
    the periodic boundary; non-neighbour beads (|i-j|>3) keep min_dist apart.
    """
    half = L / 2 - margin
    cell = min_dist
    ncell = max(1, int(L // cell))
    grid: Dict[Tuple[int, int, int], List[int]] = {}
    md2 = min_dist ** 2
    hl = L / 2

    def key(p):
        return (int((p[0] + hl) // cell) % ncell, int((p[1] + hl) // cell) % ncell,
                int((p[2] + hl) // cell) % ncell)

    def clash(p, upto):
        k = key(p)
        px, py, pz = float(p[0]), float(p[1]), float(p[2])
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    kk = ((k[0] + dx) % ncell, (k[1] + dy) % ncell, (k[2] + dz) % ncell)
                    for j in grid.get(kk, ()):
                        if j < upto - 3:
                            q = posl[j]
                            ex, ey, ez = q[0] - px, q[1] - py, q[2] - pz
                            if ex * ex + ey * ey + ez * ez < md2:
                                return True
        return False

    pos = np.zeros((n_beads, 3))
    posl = [None] * n_beads             # the same positions as Python floats
    # a walk that keeps back-tracking in a dead end is started afresh
    limit = 20 * n_beads + 10000
    iters = 0
    pos[0] = rng.uniform(-half / 2, half / 2, 3)
    d = rng.normal(size=3)
    pos[1] = pos[0] + bond * d / np.linalg.norm(d)
    for b in (0, 1):
        posl[b] = (float(pos[b][0]), float(pos[b][1]), float(pos[b][2]))
        grid.setdefault(key(pos[b]), []).append(b)
    ct = math.cos(math.radians(180.0 - theta0))
    st = math.sin(math.radians(180.0 - theta0))
    i = 2
    fails = 0
    while i < n_beads:
        iters += 1
        if iters > limit:
            return _self_avoiding_chain(rng, n_beads, L, bond, theta0, min_dist, margin)
        u = pos[i - 1] - pos[i - 2]
        u /= np.linalg.norm(u)
        a = np.cross(u, [1.0, 0.0, 0.0])
        if np.linalg.norm(a) < 1e-3:
            a = np.cross(u, [0.0, 1.0, 0.0])
        a /= np.linalg.norm(a)
        b2 = np.cross(u, a)
        ok = False
        for _ in range(40):
            phi = rng.uniform(0, 2 * np.pi)
            d = ct * u + st * (math.cos(phi) * a + math.sin(phi) * b2)
            p = pos[i - 1] + bond * d
            if np.all(np.abs(p) < half) and not clash(p, i):
                ok = True
                break
        if ok:
            pos[i] = p
            posl[i] = (float(p[0]), float(p[1]), float(p[2]))
            grid.setdefault(key(p), []).append(i)
            i += 1
            fails = 0
        else:
            # back-track a few beads
            fails += 1
            nb = min(i - 2, 2 + fails)
            for j in range(i - nb, i):
                grid[key(pos[j])].remove(j)
            i -= nb
    return pos


def solvated_chain(n_atoms: int = 23558, L: float = 62.23, n_beads: int = 2489,
                   seed: int = 1234, n_types: int = 8, name: str = "chain") -> System:
    """Seeded bead chain (bonds, angles, n=3 dihedrals, 1-4 scaled LJ) in TIP3P."""
    rng = np.random.default_rng(seed)
    n_water = (n_atoms - n_beads) // 3
    if n_beads + 3 * n_water != n_atoms:
        raise ValueError("n_atoms - n_beads must be a multiple of 3")
    chain = _self_avoiding_chain(rng, n_beads, L)
    # LJ types: eps in [0.05, 0.2], rmin/2 in [1.3, 2.1]; 1-4 values scaled
    types = [f"CB{k + 1}" for k in range(n_types)]
    eps = np.linspace(0.05, 0.2, n_types)
    rmh = np.linspace(1.3, 2.1, n_types)
    perm = rng.permutation(n_types)
    lj = {types[k]: (-float(eps[perm[k]]), float(rmh[k])) for k in range(n_types)}
    lj14 = {t: (0.5 * lj[t][0], lj[t][1] - 0.1) for t in types}
    bead_type = [types[k] for k in rng.integers(0, n_types, n_beads)]
    q = rng.uniform(-0.5, 0.5, n_beads)
    q -= q.mean()
    # waters: candidate lattice sites away from the chain
    n_edge = int(math.ceil((n_water * 1.6) ** (1.0 / 3.0)))
    sites = _lattice_sites(L, n_edge)
    # distance to nearest bead (minimum image) via a coarse cell search
    keep = np.ones(sites.shape[0], bool)
    cell = 3.0
    nc = int(L // cell)
    bins: Dict[Tuple[int, int, int], List[int]] = {}
    for j, p in enumerate(chain):
        k = tuple(((p + L / 2) // (L / nc)).astype(int) % nc)
        bins.setdefault(k, []).append(j)
    for s_i, s in enumerate(sites):
        k = ((s + L / 2) // (L / nc)).astype(int) % nc
        near = False
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    kk = ((k[0] + dx) % nc, (k[1] + dy) % nc, (k[2] + dz) % nc)
                    for j in bins.get(kk, ()):
                        d = chain[j] - s
                        d -= L * np.round(d / L)
                        if d @ d < 3.0 ** 2:
                            near = True
                            break
                    if near:
                        break
                if near:
                    break
        keep[s_i] = not near
    sites = sites[keep]
    if sites.shape[0] < n_water:
        raise RuntimeError("not enough free lattice sites for the solvent")
    sites = sites[np.sort(rng.choice(sites.shape[0], n_water, replace=False))]
    wpos = _place_waters(rng, sites, 0.2, L, others=chain, d_min=1.6)

    wb, wa, wt, wn, wrn, wri, ws = _water_topology(n_water, first_atom=n_beads)
    cb = np.stack([np.arange(n_beads - 1), np.arange(1, n_beads)], 1)
    ca = np.stack([np.arange(n_beads - 2), np.arange(1, n_beads - 1), np.arange(2, n_beads)], 1)
    cd = np.stack([np.arange(n_beads - 3), np.arange(1, n_beads - 2),
                   np.arange(2, n_beads - 1), np.arange(3, n_beads)], 1)
    wp = _water_params()
    bond_params = dict(wp["bond_params"])
    angle_params = dict(wp["angle_params"])
    dihedral_params: Dict[Tuple[str, str, str, str], List[Tuple[float, int, float]]] = {}
    for a in range(n_types):
        for b in range(a, n_types):
            bond_params[(types[a], types[b])] = (222.0, 1.53)
            dihedral_params[("X", types[a], types[b], "X")] = [(0.2, 3, 0.0)]
    for a in range(n_types):
        for b in range(n_types):
            for c in range(a, n_types):
                angle_params[(types[a], types[b], types[c])] = (58.0, 111.0)
    masses_by_type = dict(wp["masses_by_type"])
    for t in types:
        masses_by_type[t] = 12.011
    lj_all = dict(wp["lj"])
    lj_all.update(lj)
    return System(
        name=name, box=(L, L, L),
        pos=np.concatenate([chain, wpos]),
        charge=np.concatenate([q, np.tile([Q_O, Q_H, Q_H], n_water)]),
        mass=np.concatenate([np.full(n_beads, 12.011), np.tile([M_O, M_H, M_H], n_water)]),
        atom_type=bead_type + wt,
        atom_name=["CB"] * n_beads + wn,
        res_name=["BEAD"] * n_beads + wrn,
        res_id=list(range(1, n_beads + 1)) + wri,
        seg_id=["CHN"] * n_beads + ws,
        bonds=np.concatenate([cb, wb]).astype(np.int64),
        angles=np.concatenate([ca, wa]).astype(np.int64),
        dihedrals=cd.astype(np.int64), impropers=np.zeros((0, 4), np.int64),
        masses_by_type=masses_by_type, bond_params=bond_params,
        angle_params=angle_params, dihedral_params=dihedral_params,
        improper_params={}, lj_params=lj_all, lj14_params=lj14,
    )


def _dir(axis, refv, theta, phi):
    """Unit vector at angle theta (degrees) from `axis`, turned by phi
    (degrees) about it out of the plane of `axis` and `refv`."""
    u = axis / np.linalg.norm(axis)
    r = refv - (refv @ u) * u
    r /= np.linalg.norm(r)
    w = np.cross(u, r)
    t, f = math.radians(theta), math.radians(phi)
    return math.cos(t) * u + math.sin(t) * (math.cos(f) * r + math.sin(f) * w)


def _ethanol():
    """CH3-CH2-OH: SHAKE clusters of 4 (CH3), 3 (CH2) and 2 (OH) atoms."""
    c1 = np.array([0.0, 0.0, 0.0])
    c2 = np.array([1.528, 0.0, 0.0])
    o1 = c2 + 1.42 * _dir(c1 - c2, np.array([0.0, 1.0, 0.0]), 110.1, 0.0)
    h_c1 = [c1 + 1.111 * _dir(c2 - c1, o1 - c2, 110.1, 180.0 + k * 120.0) for k in range(3)]
    h_c2 = [c2 + 1.111 * _dir(c1 - c2, o1 - c2, 110.1, k) for k in (120.0, 240.0)]
    ho = o1 + 0.96 * _dir(c2 - o1, c1 - c2, 106.0, 180.0)
    return dict(
        xyz=np.stack([c1, *h_c1, c2, *h_c2, o1, ho]),
        types=["CT3", "HA", "HA", "HA", "CT2", "HA", "HA", "OH1", "H"],
        names=["C1", "H11", "H12", "H13", "C2", "H21", "H22", "O1", "HO1"],
        charges=[-0.27, 0.09, 0.09, 0.09, 0.05, 0.09, 0.09, -0.66, 0.43],
        bonds=[(0, 1), (0, 2), (0, 3), (0, 4), (4, 5), (4, 6), (4, 7), (7, 8)],
        resname="ETOH")


def _glycol():
    """HO-CH2-CH2-OH: SHAKE clusters of 3 (CH2) and 2 (OH) atoms only."""
    c1 = np.array([0.0, 0.0, 0.0])
    c2 = np.array([1.53, 0.0, 0.0])
    o1 = c1 + 1.42 * _dir(c2 - c1, np.array([0.0, 1.0, 0.0]), 110.1, 0.0)
    o2 = c2 + 1.42 * _dir(c1 - c2, o1 - c1, 110.1, 180.0)
    h_c1 = [c1 + 1.111 * _dir(c2 - c1, o1 - c1, 110.1, k) for k in (120.0, 240.0)]
    h_c2 = [c2 + 1.111 * _dir(c1 - c2, o2 - c2, 110.1, k) for k in (120.0, 240.0)]
    ho1 = o1 + 0.96 * _dir(c1 - o1, c2 - c1, 106.0, 180.0)
    ho2 = o2 + 0.96 * _dir(c2 - o2, c1 - c2, 106.0, 180.0)
    return dict(
        xyz=np.stack([o1, ho1, c1, *h_c1, c2, *h_c2, o2, ho2]),
        types=["OH1", "H", "CT2", "HA", "HA", "CT2", "HA", "HA", "OH1", "H"],
        names=["O1", "HO1", "C1", "H11", "H12", "C2", "H21", "H22", "O2", "HO2"],
        charges=[-0.66, 0.43, 0.05, 0.09, 0.09, 0.05, 0.09, 0.09, -0.66, 0.43],
        bonds=[(0, 1), (0, 2), (2, 3), (2, 4), (2, 5), (5, 6), (5, 7), (5, 8), (8, 9)],
        resname="EGLY")


def _angles_dihedrals(bonds, n):
    """All angles i-j-k and proper dihedrals i-j-k-l of a bond graph."""
    nb = [set() for _ in range(n)]
    for a, b in bonds:
        nb[a].add(b)
        nb[b].add(a)
    angles = sorted({(min(i, k), j, max(i, k)) for j in range(n) for i in nb[j] for k in nb[j] if i != k})
    dih = set()
    for j, k in bonds:
        for i in nb[j] - {k}:
            for l in nb[k] - {j}:
                if i != l:
                    dih.add((i, j, k, l) if (i, j) < (l, k) else (l, k, j, i))
    return angles, sorted(dih)


# CHARMM-like parameters of the small solutes (types CT3, CT2, HA, OH1, H)
_SOLUTE_BONDS = {("CT3", "HA"): (322.0, 1.111), ("CT2", "HA"): (309.0, 1.111),
                 ("CT2", "CT3"): (222.5, 1.528), ("CT2", "CT2"): (222.5, 1.53),
                 ("CT2", "OH1"): (428.0, 1.42), ("H", "OH1"): (545.0, 0.96)}
_SOLUTE_ANGLES = {("HA", "CT3", "HA"): (35.5, 108.4), ("CT2", "CT3", "HA"): (34.6, 110.1),
                  ("CT3", "CT2", "HA"): (34.6, 110.1), ("HA", "CT2", "HA"): (35.5, 109.0),
                  ("CT3", "CT2", "OH1"): (75.7, 110.1), ("HA", "CT2", "OH1"): (45.9, 108.89),
                  ("CT2", "OH1", "H"): (57.5, 106.0), ("CT2", "CT2", "HA"): (26.5, 110.1),
                  ("CT2", "CT2", "OH1"): (75.7, 110.1)}
_SOLUTE_DIHEDRALS = {("X", "CT2", "CT3", "X"): [(0.16, 3, 0.0)],
                     ("X", "CT2", "OH1", "X"): [(0.14, 3, 0.0)],
                     ("X", "CT2", "CT2", "X"): [(0.19, 3, 0.0)]}
_SOLUTE_LJ = {"CT3": (-0.078, 2.04), "CT2": (-0.055, 2.175), "HA": (-0.022, 1.32),
              "OH1": (-0.1521, 1.77), "H": (-0.046, 0.2245)}
_SOLUTE_MASSES = {"CT3": 12.011, "CT2": 12.011, "HA": 1.008, "OH1": 15.999, "H": 1.008}


def solvated_solute(mol: dict, n_mol: int, L: float, seed: int, name: str) -> System:
    """n_mol copies of a small molecule at seeded random positions (at least
    6.5 A apart) and orientations in a TIP3P box of edge L, waters on a
    jittered lattice away from the solutes."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    t = mol["xyz"] - mol["xyz"].mean(axis=0)
    na = t.shape[0]
    R = _random_rotations(rng, n_mol)
    centres = []
    while len(centres) < n_mol:
        c = rng.uniform(-L / 2, L / 2, 3)
        if all(np.linalg.norm((c - q) - L * np.round((c - q) / L)) > 6.5 for q in centres):
            centres.append(c)
    spos = (np.asarray(centres)[:, None, :] + np.einsum("nij,aj->nai", R, t)).reshape(-1, 3)

    def _wrap(p):
        w = np.mod(p + L / 2, L)
        return np.where(w >= L, w - L, w)
    sites = _lattice_sites(L, int(round(L / 3.0)))
    dist, _ = cKDTree(_wrap(spos), boxsize=L).query(_wrap(sites), k=1)
    sites = sites[dist >= 2.7]
    n_water = sites.shape[0]
    wpos = _place_waters(rng, sites, 0.2, L, others=spos, d_min=1.6)
    ns = na * n_mol
    wb, wa, wt, wn, wrn, wri, ws = _water_topology(n_water, first_atom=ns, first_res=n_mol + 1)
    ang1, dih1 = _angles_dihedrals(mol["bonds"], na)
    off = (na * np.arange(n_mol))[:, None, None]
    b = (np.asarray(mol["bonds"])[None] + off).reshape(-1, 2)
    a = (np.asarray(ang1)[None] + off).reshape(-1, 3)
    d = (np.asarray(dih1)[None] + off).reshape(-1, 4)
    wp = _water_params()
    bond_params = {**wp["bond_params"], **_SOLUTE_BONDS}
    angle_params = {**wp["angle_params"], **_SOLUTE_ANGLES}
    masses = {**wp["masses_by_type"], **_SOLUTE_MASSES}
    lj = {**wp["lj"], **_SOLUTE_LJ}
    types = mol["types"] * n_mol + wt
    return System(
        name=name, box=(L, L, L), pos=np.concatenate([spos, wpos]),
        charge=np.concatenate([np.tile(mol["charges"], n_mol), np.tile([Q_O, Q_H, Q_H], n_water)]),
        mass=np.array([masses[x] for x in types]),
        atom_type=types, atom_name=mol["names"] * n_mol + wn,
        res_name=[mol["resname"]] * ns + wrn,
        res_id=[1 + k // na for k in range(ns)] + wri,
        seg_id=["SOL"] * ns + ws,
        bonds=np.concatenate([b, wb]).astype(np.int64),
        angles=np.concatenate([a, wa]).astype(np.int64),
        dihedrals=d.astype(np.int64), impropers=np.zeros((0, 4), np.int64),
        masses_by_type=masses, bond_params=bond_params, angle_params=angle_params,
        dihedral_params=dict(_SOLUTE_DIHEDRALS), improper_params={}, lj_params=lj,
        lj14_params={},
    )


# --------------------------------------------------------------------------
# named workloads
# --------------------------------------------------------------------------

def config_small_water(seed: int = 2024) -> System:
    """12,480-atom TIP3P box, 50 A edge; PME 48^3 order 4, roff 10, ron 8, list 12."""
    s = water_box(4160, 50.0, seed=seed, name="water12k")
    s.settings = dict(kappa=0.34, nfft=(48, 48, 48), order=4, ctofnb=10.0,
                      ctonnb=8.0, cutnb=12.0, dt_ps=0.002)
    return s


def config_solvated_chain(seed: int = 1234) -> System:
    """23,558-atom bead chain in TIP3P, 62.23 A; PME 64^3 order 6, roff 12, ron 10, list 14."""
    s = solvated_chain(seed=seed, name="chain23k")
    s.settings = dict(kappa=0.34, nfft=(64, 64, 64), order=6, ctofnb=12.0,
                      ctonnb=10.0, cutnb=14.0, dt_ps=0.002)
    return s


def config_large_water(seed: int = 77) -> System:
    """~1M-atom TIP3P box (333,333 molecules, ~215 A); PME 216^3 order 4."""
    L = (999999 / 0.1003) ** (1.0 / 3.0)
    s = water_box(333333, L, seed=seed, name="water1m")
    s.settings = dict(kappa=0.34, nfft=(216, 216, 216), order=4, ctofnb=10.0,
                      ctonnb=8.0, cutnb=11.5, dt_ps=0.002)
    return s


def config_ethanol(seed: int = 31) -> System:
    """40 ethanols in TIP3P (32 A box): SHAKE clusters of 2, 3 and 4 atoms
    beside SETTLE waters; PME 32^3 order 4, roff 10, ron 8, list 12."""
    s = solvated_solute(_ethanol(), 40, 32.0, seed, "ethanol3k")
    s.settings = dict(kappa=0.34, nfft=(32, 32, 32), order=4, ctofnb=10.0,
                      ctonnb=8.0, cutnb=12.0, dt_ps=0.002)
    return s


def config_glycol(seed: int = 37) -> System:
    """40 ethylene glycols in TIP3P (32 A box): SHAKE clusters of 2 and 3
    atoms beside SETTLE waters; PME 32^3 order 4, roff 10, ron 8, list 12."""
    s = solvated_solute(_glycol(), 40, 32.0, seed, "glycol3k")
    s.settings = dict(kappa=0.34, nfft=(32, 32, 32), order=4, ctofnb=10.0,
                      ctonnb=8.0, cutnb=12.0, dt_ps=0.002)
    return s


def batch_system(seed: int, n_atoms: int) -> System:
    """One system of the many-system workload: a bead chain of ~10 % of the
    atoms in TIP3P, the cubic box sized to 0.997 g/cm^3, PME grid spacing at
    most 1 A rounded up to an FFT-friendly size, spline order 4, cutoff 10 A
    (switch 8-10 A, list 12 A)."""
    n_beads = max(30, int(round(0.1 * n_atoms)))
    n_beads += (n_atoms - n_beads) % 3          # the rest is whole waters
    masses = n_beads * 12.011 + (n_atoms - n_beads) // 3 * (15.9994 + 2 * 1.008)
    L = (masses / (0.997 / 1.66053906660)) ** (1.0 / 3.0)
    s = solvated_chain(n_atoms=n_atoms, L=L, n_beads=n_beads, seed=seed,
                       name=f"batch{seed}")
    n = fft_friendly(int(math.ceil(L)))
    s.settings = dict(kappa=0.34, nfft=(n, n, n), order=4, ctofnb=10.0, ctonnb=8.0,
                      cutnb=12.0, dt_ps=0.002)
    return s


def batch_sizes(n_systems: int = 256, lo: int = 3000, hi: int = 30000, seed: int = 99):
    """Atom counts log-uniform in [lo, hi], seeded."""
    rng = np.random.default_rng(seed)
    return [int(v) for v in np.exp(rng.uniform(math.log(lo), math.log(hi), n_systems))]


def fft_friendly(n: int) -> int:
    """Smallest even m >= n whose prime factors are 2, 3, 5 and 7."""
    m = max(2, n)
    while True:
        if m % 2 == 0:
            k = m
            for p in (2, 3, 5, 7):
                while k % p == 0:
                    k //= p
            if k == 1:
                return m
        m += 1


# --------------------------------------------------------------------------
# CHARMM file writers
# --------------------------------------------------------------------------

def write_psf(sys: System, path: str) -> None:
    n = sys.n_atoms
    lines = ["PSF CMAP CHEQ XPLOR", "", "       2 !NTITLE",
             f"* SYNTHETIC SYSTEM {sys.name}", "* GENERATED BY apocharmm_b200.systems", "",
             f"{n:8d} !NATOM"]
    for i in range(n):
        lines.append(
            f"{i + 1:8d} {sys.seg_id[i]:<4s} {sys.res_id[i]:<4d} {sys.res_name[i]:<4s} "
            f"{sys.atom_name[i]:<4s} {sys.atom_type[i]:<4s} {sys.charge[i]:14.6f}"
            f"{sys.mass[i]:14.4f}           0   0.00000     -0.301140E-02")
    lines.append("")

    def block(arr, per_line, title):
        out = ["", f"{arr.shape[0]:8d} !{title}"]
        flat = (arr + 1).reshape(-1)
        w = arr.shape[1] if arr.ndim == 2 and arr.shape[0] else 1
        per = per_line * w
        for k in range(0, flat.size, per):
            out.append("".join(f"{v:8d}" for v in flat[k:k + per]))
        return out

    lines += block(sys.bonds, 4, "NBOND: bonds")
    lines += block(sys.angles, 3, "NTHETA: angles")
    lines += block(sys.dihedrals, 2, "NPHI: dihedrals")
    lines += block(sys.impropers, 2, "NIMPHI: impropers")
    lines += ["", "       0 !NDON: donors", "", "", "       0 !NACC: acceptors", "", "",
              "       0 !NNB", "", "", "       0       0 !NGRP NST2", "", "",
              "       0       0 !NUMLP NUMLPH", "", "       0 !NCRTERM: cross-terms", ""]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_crd(sys: System, path: str, pos: np.ndarray | None = None) -> None:
    pos = sys.pos if pos is None else pos
    n = sys.n_atoms
    ext = n >= 100000
    lines = [f"* SYNTHETIC SYSTEM {sys.name}", "*"]
    lines.append(f"{n:10d}  EXT" if ext else f"{n:5d}")
    for i in range(n):
        x, y, z = pos[i]
        if ext:
            lines.append(f"{i + 1:10d}{sys.res_id[i]:10d}  {sys.res_name[i]:<8s}  {sys.atom_name[i]:<8s}"
                         f"{x:20.10f}{y:20.10f}{z:20.10f}  {sys.seg_id[i]:<8s}  {sys.res_id[i]:<8d}{0.0:20.10f}")
        else:
            lines.append(f"{i + 1:5d}{sys.res_id[i]:5d} {sys.res_name[i]:<4s} {sys.atom_name[i]:<4s}"
                         f"{x:10.5f}{y:10.5f}{z:10.5f} {sys.seg_id[i]:<4s} {sys.res_id[i]:<4d}{0.0:10.5f}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_prm(sys: System, path: str) -> None:
    L = ["* PARAMETERS FOR SYNTHETIC SYSTEM", "*", "", "ATOMS"]
    for t, m in sys.masses_by_type.items():
        L.append(f"MASS  -1  {t:<6s} {m:10.5f}")
    L += ["", "BONDS"]
    for (a, b), (k, r0) in sys.bond_params.items():
        L.append(f"{a:<6s} {b:<6s} {k:10.4f} {r0:10.5f}")
    L += ["", "ANGLES"]
    for (a, b, c), (k, t0) in sys.angle_params.items():
        L.append(f"{a:<6s} {b:<6s} {c:<6s} {k:10.4f} {t0:10.4f}")
    L += ["", "DIHEDRALS"]
    for (a, b, c, d), terms in sys.dihedral_params.items():
        for (k, n, dl) in terms:
            L.append(f"{a:<6s} {b:<6s} {c:<6s} {d:<6s} {k:10.4f} {n:3d} {dl:10.4f}")
    L += ["", "IMPROPER"]
    for (a, b, c, d), (k, p0) in sys.improper_params.items():
        L.append(f"{a:<6s} {b:<6s} {c:<6s} {d:<6s} {k:10.4f}   0 {p0:10.4f}")
    L += ["", "NONBONDED nbxmod  5 atom cdiel fshift vatom vdistance vfswitch -",
          "cutnb 14.0 ctofnb 12.0 ctonnb 10.0 eps 1.0 e14fac 1.0 wmin 1.5", ""]
    for t, (e, rh) in sys.lj_params.items():
        if t in sys.lj14_params:
            e14, r14 = sys.lj14_params[t]
            L.append(f"{t:<6s} 0.0 {e:10.6f} {rh:10.6f} 0.0 {e14:10.6f} {r14:10.6f}")
        else:
            L.append(f"{t:<6s} 0.0 {e:10.6f} {rh:10.6f}")
    L += ["", "END", ""]
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def write_charmm_files(sys: System, directory: str) -> Dict[str, str]:
    os.makedirs(directory, exist_ok=True)
    paths = {k: os.path.join(directory, f"{sys.name}.{k}") for k in ("psf", "crd", "prm")}
    write_psf(sys, paths["psf"])
    write_crd(sys, paths["crd"])
    write_prm(sys, paths["prm"])
    return paths
