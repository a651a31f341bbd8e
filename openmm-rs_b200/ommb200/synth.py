"""Seeded synthetic inputs with the shapes of the benchmark workloads.

No public dataset is involved; every system is generated from a seed:

* ``water_box``: rigid 3-site water (O-H 0.09572 nm, H-O-H 104.52 deg, O -0.834 e,
  H +0.417 e, LJ on O only: sigma 0.315061 nm, epsilon 0.636386 kJ/mol; masses O 15.9994,
  H 1.008 Da).  Oxygens sit on a jittered lattice (uniform +-0.02 nm) with a uniformly random
  orientation per molecule.  Presets: 648 waters in a 2.70 nm box (9x9x8 lattice), 7,986
  waters in a 6.20 nm box (a seeded subset of a 20^3 lattice), 355,000 waters in a 22.0 nm
  box (a seeded subset of a 71^3 lattice).
* ``chain``: self-avoiding random walk (bond 0.153 nm, angle 109.5 deg, random dihedral,
  rejection of non-bonded contacts closer than 0.3 nm) with neutralised N(0, 0.3) charges,
  LJ sigma 0.30 nm / epsilon 0.40 kJ/mol and OBC radii uniform in [0.12, 0.20] nm, scale 0.8.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import math

import numpy as np

D_OH = 0.09572
ANGLE_HOH = np.deg2rad(104.52)
D_HH = 2.0 * D_OH * np.sin(0.5 * ANGLE_HOH)
MASS_O, MASS_H = 15.9994, 1.008
Q_O, Q_H = -0.834, 0.417
SIGMA_O, EPS_O = 0.315061, 0.636386


@dataclass
class WaterBox:
    positions: np.ndarray  # [3*nw, 3] nm, order O,H,H per molecule
    box: np.ndarray  # [3,3] row vectors
    n_waters: int

    @property
    def n_atoms(self) -> int:
        return 3 * self.n_waters

    def masses(self) -> np.ndarray:
        return np.tile([MASS_O, MASS_H, MASS_H], self.n_waters)

    def charges(self) -> np.ndarray:
        return np.tile([Q_O, Q_H, Q_H], self.n_waters)

    def sigmas(self) -> np.ndarray:
        return np.tile([SIGMA_O, 1.0, 1.0], self.n_waters)

    def epsilons(self) -> np.ndarray:
        return np.tile([EPS_O, 0.0, 0.0], self.n_waters)

    def exceptions(self):
        """Three exclusions per water (chargeProd 0, epsilon 0)."""
        out = []
        for w in range(self.n_waters):
            o = 3 * w
            out += [(o, o + 1, 0.0, 1.0, 0.0), (o, o + 2, 0.0, 1.0, 0.0),
                    (o + 1, o + 2, 0.0, 1.0, 0.0)]
        return out

    def constraints(self):
        out = []
        for w in range(self.n_waters):
            o = 3 * w
            out += [(o, o + 1, D_OH), (o, o + 2, D_OH), (o + 1, o + 2, D_HH)]
        return out

    def waters(self) -> np.ndarray:
        return np.arange(3 * self.n_waters, dtype=np.int32).reshape(-1, 3)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from uniform unit quaternions (Shoemake 1992)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a = np.sqrt(1 - u1)
    b = np.sqrt(u1)
    qw = a * np.sin(2 * np.pi * u2)
    qx = a * np.cos(2 * np.pi * u2)
    qy = b * np.sin(2 * np.pi * u3)
    qz = b * np.cos(2 * np.pi * u3)
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (qy * qy + qz * qz)
    r[:, 0, 1] = 2 * (qx * qy - qz * qw)
    r[:, 0, 2] = 2 * (qx * qz + qy * qw)
    r[:, 1, 0] = 2 * (qx * qy + qz * qw)
    r[:, 1, 1] = 1 - 2 * (qx * qx + qz * qz)
    r[:, 1, 2] = 2 * (qy * qz - qx * qw)
    r[:, 2, 0] = 2 * (qx * qz - qy * qw)
    r[:, 2, 1] = 2 * (qy * qz + qx * qw)
    r[:, 2, 2] = 1 - 2 * (qx * qx + qy * qy)
    return r


def water_box(n_waters: int, box_length: float, lattice, seed: int = 2024,
              jitter: float = 0.02) -> WaterBox:
    """Rigid water on a jittered lattice; `lattice` = (nx, ny, nz) sites, of which a seeded
    random subset of `n_waters` is occupied."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = lattice
    sites = nx * ny * nz
    if n_waters > sites:
        raise ValueError("more waters than lattice sites")
    idx = np.arange(sites) if n_waters == sites else np.sort(rng.choice(sites, n_waters, replace=False))
    ix, iy, iz = idx // (ny * nz), (idx // nz) % ny, idx % nz
    spacing = np.array([box_length / nx, box_length / ny, box_length / nz])
    o = (np.stack([ix, iy, iz], 1) + 0.5) * spacing
    o += rng.uniform(-jitter, jitter, size=o.shape)
    # canonical geometry: O at the origin, H in the xy plane symmetric about y
    h = np.array([[D_OH * np.sin(ANGLE_HOH / 2), D_OH * np.cos(ANGLE_HOH / 2), 0.0],
                  [-D_OH * np.sin(ANGLE_HOH / 2), D_OH * np.cos(ANGLE_HOH / 2), 0.0]])
    rot = _random_rotations(rng, n_waters)
    hpos = np.einsum("nij,kj->nki", rot, h) + o[:, None, :]
    pos = np.empty((n_waters, 3, 3))
    pos[:, 0] = o
    pos[:, 1:] = hpos
    box = np.diag([box_length] * 3).astype(np.float64)
    return WaterBox(positions=pos.reshape(-1, 3), box=box, n_waters=n_waters)


WATER_PRESETS = {
    "water-1944": dict(n_waters=648, box_length=2.70, lattice=(9, 9, 8)),
    "water-23958": dict(n_waters=7986, box_length=6.20, lattice=(20, 20, 20)),
    "water-1065000": dict(n_waters=355000, box_length=22.0, lattice=(71, 71, 71)),
}


def water_preset(name: str, seed: int = 2024) -> WaterBox:
    return water_box(seed=seed, **WATER_PRESETS[name])


@dataclass
class Chain:
    positions: np.ndarray
    charges: np.ndarray
    sigma: float = 0.30
    epsilon: float = 0.40
    radii: np.ndarray = field(default_factory=lambda: np.zeros(0))
    gb_scale: float = 0.8
    bond_length: float = 0.153
    bond_k: float = 2.5e5
    angle: float = float(np.deg2rad(109.5))
    angle_k: float = 400.0
    mass: float = 12.011

    @property
    def n_atoms(self) -> int:
        return len(self.positions)

    def bonds(self):
        return [(i, i + 1, self.bond_length, self.bond_k) for i in range(self.n_atoms - 1)]

    def angles(self):
        return [(i, i + 1, i + 2, self.angle, self.angle_k) for i in range(self.n_atoms - 2)]


def chain(n_atoms: int, seed: int, min_contact: float = 0.3, max_tries: int = 200) -> Chain:
    """Self-avoiding random walk with tetrahedral bond angles and random dihedrals: monomer i
    keeps at least `min_contact` from every monomer before i - 3 (checked on a cell grid of
    that width); a monomer with no valid dihedral after `max_tries` draws backs the walk up
    five monomers."""
    rng = np.random.default_rng(seed)
    b = 0.153
    theta = np.deg2rad(109.5)
    cos_t, sin_t = math.cos(theta), math.sin(theta)
    mc2 = min_contact * min_contact
    pos = [(0.0, 0.0, 0.0)] * n_atoms
    if n_atoms > 1:
        pos[1] = (b, 0.0, 0.0)
    if n_atoms > 2:
        pos[2] = (b - b * cos_t, b * sin_t, 0.0)
    cells = {}
    in_grid = 0  # monomers 0 .. in_grid-1 are on the grid

    def cell(p):
        return (math.floor(p[0] / min_contact), math.floor(p[1] / min_contact),
                math.floor(p[2] / min_contact))

    def clear(p, i):
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in cells.get((p[0] + dx, p[1] + dy, p[2] + dz), ()):
                        q = pos[j]
                        ex, ey, ez = q[0] - i[0], q[1] - i[1], q[2] - i[2]
                        if ex * ex + ey * ey + ez * ez < mc2:
                            return False
        return True

    i = 3
    restarts = 0
    while i < n_atoms:
        while in_grid < i - 3:
            cells.setdefault(cell(pos[in_grid]), []).append(in_grid)
            in_grid += 1
        a, bb, c = pos[i - 3], pos[i - 2], pos[i - 1]
        bc = (c[0] - bb[0], c[1] - bb[1], c[2] - bb[2])
        nb = math.sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2])
        bc = (bc[0] / nb, bc[1] / nb, bc[2] / nb)
        u = (bb[0] - a[0], bb[1] - a[1], bb[2] - a[2])
        nrm = (u[1] * bc[2] - u[2] * bc[1], u[2] * bc[0] - u[0] * bc[2], u[0] * bc[1] - u[1] * bc[0])
        nn = math.sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2])
        nrm = (nrm[0] / nn, nrm[1] / nn, nrm[2] / nn)
        m = (nrm[1] * bc[2] - nrm[2] * bc[1], nrm[2] * bc[0] - nrm[0] * bc[2],
             nrm[0] * bc[1] - nrm[1] * bc[0])
        placed = False
        for _ in range(max_tries):
            phi = rng.uniform(-np.pi, np.pi)
            d0, d1, d2 = -b * cos_t, b * sin_t * math.cos(phi), b * sin_t * math.sin(phi)
            p = tuple(c[k] + d0 * bc[k] + d1 * m[k] + d2 * nrm[k] for k in range(3))
            if in_grid and not clear(cell(p), p):
                continue
            pos[i] = p
            placed = True
            break
        if placed:
            i += 1
        else:  # dead end: back up a few monomers
            restarts += 1
            i = max(3, i - 5)
            while in_grid > i - 3:
                in_grid -= 1
                cells[cell(pos[in_grid])].remove(in_grid)
            if restarts > 100 * n_atoms:
                raise RuntimeError("self-avoiding walk failed")
    pos = np.array(pos, dtype=np.float64).reshape(n_atoms, 3)
    pos -= pos.mean(axis=0)
    q = rng.normal(0.0, 0.3, n_atoms)
    q -= q.mean()
    radii = rng.uniform(0.12, 0.20, n_atoms)
    return Chain(positions=pos, charges=q, radii=radii)


def chain_batch(n_chains: int = 256, lo: int = 200, hi: int = 2000, seed: int = 7):
    """Chains with sizes uniform in [lo, hi] drawn from `seed`."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, n_chains)
    return [chain(int(s), seed=seed * 100003 + k) for k, s in enumerate(sizes)]
