"""Molecules and seeded synthetic geometries for the DF workloads.

``Molecule`` keeps the fields of the reference's container
(``asuka/frontend/molecule.py:51-94``: atoms in bohr, charge, spin, basis name,
Cartesian flag) that the DF path reads.  The generators restate the workload
definitions: N2 at 1.0977 A, seeded water clusters (O-H 0.9572 A,
HOH 104.52 deg, random orientation from the QR of a standard-normal 3x3, O
sites uniform in a cube of edge max(3, (30 n)^(1/3)) A with rejection at
O-O < 2.7 A) and a seeded all-trans n-decane.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .basis import ATOMIC_NUMBER

ANGSTROM_TO_BOHR = 1.8897259886  # asuka/frontend/molecule.py:9


@dataclass(frozen=True)
class Molecule:
    atoms_bohr: tuple[tuple[str, np.ndarray], ...]
    charge: int = 0
    spin: int = 0
    basis: str | None = None
    cart: bool = True

    @classmethod
    def from_atoms(cls, atoms, *, unit: str = "Bohr", charge: int = 0, spin: int = 0,
                   basis: str | None = None, cart: bool = True) -> "Molecule":
        if isinstance(atoms, str):
            parsed = []
            for frag in atoms.replace("\n", ";").split(";"):
                tok = frag.split()
                if not tok:
                    continue
                if len(tok) != 4:
                    raise ValueError(f"invalid atom fragment: {frag!r}")
                parsed.append((tok[0], np.array([float(t) for t in tok[1:]])))
            atoms = parsed
        u = unit.strip().lower()
        if u in ("bohr", "a0", "au"):
            s = 1.0
        elif u in ("angstrom", "ang", "a"):
            s = ANGSTROM_TO_BOHR
        else:
            raise ValueError("unit must be 'Bohr' or 'Angstrom'")
        ab = tuple((str(el), np.asarray(xyz, dtype=np.float64).reshape(3) * s) for el, xyz in atoms)
        if not ab:
            raise ValueError("no atoms")
        return cls(atoms_bohr=ab, charge=int(charge), spin=int(spin), basis=basis, cart=bool(cart))

    @property
    def natm(self) -> int:
        return len(self.atoms_bohr)

    @property
    def elements(self) -> tuple[str, ...]:
        return tuple(el for el, _ in self.atoms_bohr)

    @property
    def coords_bohr(self) -> np.ndarray:
        return np.asarray([xyz for _, xyz in self.atoms_bohr], dtype=np.float64).reshape((-1, 3))

    @property
    def charges(self) -> np.ndarray:
        return np.asarray([ATOMIC_NUMBER[el] for el in self.elements], dtype=np.float64)

    @property
    def nelectron(self) -> int:
        return int(round(self.charges.sum())) - int(self.charge)

    def with_coords(self, coords_bohr: np.ndarray) -> "Molecule":
        R = np.asarray(coords_bohr, dtype=np.float64).reshape((self.natm, 3))
        return Molecule(tuple((el, R[i].copy()) for i, el in enumerate(self.elements)),
                        self.charge, self.spin, self.basis, self.cart)

    def energy_nuc(self) -> float:
        Z, R = self.charges, self.coords_bohr
        e = 0.0
        for i in range(self.natm):
            for j in range(i):
                e += Z[i] * Z[j] / float(np.linalg.norm(R[i] - R[j]))
        return e

    def energy_nuc_grad(self) -> np.ndarray:
        """dE_nuc/dR, (natm, 3) in Eh/bohr (``asuka/frontend/molecule.py:148``)."""
        Z, R = self.charges, self.coords_bohr
        d = R[:, None, :] - R[None, :, :]
        r = np.sqrt((d * d).sum(-1))
        np.fill_diagonal(r, np.inf)
        f = -(Z[:, None] * Z[None, :]) / r**3
        return (f[:, :, None] * d).sum(1)


def n2(basis: str = "ma-svp", r_angstrom: float = 1.0977) -> Molecule:
    return Molecule.from_atoms([("N", (0, 0, 0)), ("N", (0, 0, r_angstrom))], unit="Angstrom", basis=basis)


def water(basis: str = "ma-svp") -> Molecule:
    r, th = 0.9572, np.deg2rad(104.52)
    return Molecule.from_atoms(
        [("O", (0, 0, 0)), ("H", (r, 0, 0)), ("H", (r * np.cos(th), r * np.sin(th), 0))],
        unit="Angstrom", basis=basis)


def water_cluster(n: int, seed: int, basis: str = "ma-tzvp") -> Molecule:
    """Seeded (H2O)_n: O uniform in a cube, min O-O 2.7 A, random rigid orientations."""
    rng = np.random.default_rng(seed)
    edge = max(3.0, (30.0 * n) ** (1.0 / 3.0))
    oxy: list[np.ndarray] = []
    while len(oxy) < n:
        p = rng.uniform(0.0, edge, 3)
        if all(np.linalg.norm(p - q) >= 2.7 for q in oxy):
            oxy.append(p)
    r, th = 0.9572, np.deg2rad(104.52)
    h1 = np.array([r, 0.0, 0.0])
    h2 = np.array([r * np.cos(th), r * np.sin(th), 0.0])
    atoms = []
    for o in oxy:
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        atoms += [("O", o), ("H", o + q @ h1), ("H", o + q @ h2)]
    return Molecule.from_atoms(atoms, unit="Angstrom", basis=basis)


def decane(seed: int = 0, basis: str = "ma-svp", jitter: float = 0.05) -> Molecule:
    """All-trans n-C10H22 (C-C 1.53 A, C-H 1.09 A, tetrahedral angles) with seeded U(+-jitter) noise."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.53, 1.09
    tet = np.arccos(-1.0 / 3.0)
    half = tet / 2.0
    # zig-zag backbone in the xy plane
    carbons = [np.array([i * cc * np.sin(half), (i % 2) * cc * np.cos(half), 0.0]) for i in range(10)]
    atoms: list[tuple[str, np.ndarray]] = []
    for i, c in enumerate(carbons):
        atoms.append(("C", c))
        nbrs = [carbons[j] for j in (i - 1, i + 1) if 0 <= j < 10]
        u = sum((c - b) / np.linalg.norm(c - b) for b in nbrs)
        u = u / np.linalg.norm(u)
        if len(nbrs) == 2:
            # two H in the plane perpendicular to the C-C-C plane, bisected by u
            ang = tet / 2.0
            for sgn in (1.0, -1.0):
                v = np.cos(ang) * u + np.sin(ang) * np.array([0.0, 0.0, sgn])
                atoms.append(("H", c + ch * v / np.linalg.norm(v)))
        else:
            # terminal CH3: staggered around the C-C axis
            axis = u
            perp = np.cross(axis, np.array([0.0, 0.0, 1.0]))
            perp /= np.linalg.norm(perp)
            perp2 = np.cross(axis, perp)
            for k in range(3):
                phi = 2.0 * np.pi * k / 3.0
                v = np.cos(np.pi - tet) * axis + np.sin(np.pi - tet) * (np.cos(phi) * perp2 + np.sin(phi) * perp)
                atoms.append(("H", c + ch * v))
    out = [(el, xyz + rng.uniform(-jitter, jitter, 3)) for el, xyz in atoms]
    return Molecule.from_atoms(out, unit="Angstrom", basis=basis)
