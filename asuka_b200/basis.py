"""Packed Cartesian Gaussian bases and shell pairs.

Mirrors the reference's packed structure-of-arrays basis
(``asuka/cueri/basis_cart.py:12`` ``BasisCartSoA``) and its l-ordered shell-pair
list (``asuka/cueri/shell_pairs.py:72`` ``build_shell_pairs_l_order``), so the
same arrays can be handed to the DF engine whichever side built them.

Conventions (identical to the reference):

* every shell is one contraction column (contractions expanded,
  ``asuka/frontend/basis_packer.py:210-238``); ``prim_coef`` already holds the
  Cartesian normalisation (``asuka/integrals/gto_cart.py:54-66``);
* Cartesian component order inside a shell is x-major,
  ``for x = l..0: for y = l-x..0: z = l-x-y``;
* AO functions of shell ``s`` occupy ``shell_ao_start[s] : +ncart(l)``.

Per-element shell data (AO basis and RICD acCD aux basis) come from
``data/basis_tables.npz``, produced by ``data/make_basis_tables.py``.
"""

from __future__ import annotations

import functools
import os
from dataclasses import dataclass

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

ATOMIC_NUMBER = {"H": 1, "He": 2, "C": 6, "N": 7, "O": 8, "F": 9}


def ncart(l: int) -> int:
    return (int(l) + 1) * (int(l) + 2) // 2


def cart_components(l: int) -> np.ndarray:
    """(ncart(l), 3) int array of (lx, ly, lz) in the x-major order."""
    out = []
    for x in range(l, -1, -1):
        for y in range(l - x, -1, -1):
            out.append((x, y, l - x - y))
    return np.asarray(out, dtype=np.int32).reshape((-1, 3))


@dataclass(frozen=True)
class BasisCartSoA:
    """Structure-of-arrays Cartesian basis (field names follow the reference)."""

    shell_cxyz: np.ndarray  # (nshell, 3) float64, bohr
    shell_prim_start: np.ndarray  # (nshell,) int32
    shell_nprim: np.ndarray  # (nshell,) int32
    shell_l: np.ndarray  # (nshell,) int32
    shell_ao_start: np.ndarray  # (nshell,) int32
    prim_exp: np.ndarray  # (nprim,) float64
    prim_coef: np.ndarray  # (nprim,) float64
    shell_atom: np.ndarray | None = None  # (nshell,) int32, owning atom

    def __post_init__(self) -> None:
        n = int(self.shell_l.shape[0])
        if self.shell_cxyz.shape != (n, 3) or self.shell_cxyz.dtype != np.float64:
            raise ValueError("shell_cxyz must be float64 with shape (nshell, 3)")
        for name in ("shell_prim_start", "shell_nprim", "shell_l", "shell_ao_start"):
            a = getattr(self, name)
            if a.dtype != np.int32 or a.shape != (n,):
                raise ValueError(f"{name} must be int32 with shape (nshell,)")
        if self.prim_exp.dtype != np.float64 or self.prim_coef.shape != self.prim_exp.shape:
            raise ValueError("prim_exp/prim_coef must be float64 arrays of equal length")

    @property
    def nshell(self) -> int:
        return int(self.shell_l.shape[0])

    @property
    def nao(self) -> int:
        if self.nshell == 0:
            return 0
        return int(self.shell_ao_start[-1]) + ncart(int(self.shell_l[-1]))

    @property
    def lmax(self) -> int:
        return int(self.shell_l.max()) if self.nshell else 0


@dataclass(frozen=True)
class ShellPairs:
    """Unique unordered shell pairs oriented so that l(A) >= l(B)."""

    sp_A: np.ndarray
    sp_B: np.ndarray
    sp_npair: np.ndarray
    sp_pair_start: np.ndarray

    @property
    def nsp(self) -> int:
        return int(self.sp_A.shape[0])


@functools.lru_cache(maxsize=1)
def _tables() -> dict[str, np.ndarray]:
    with np.load(os.path.join(_DATA, "basis_tables.npz")) as z:
        return {k: z[k] for k in z.files}


def available_bases() -> tuple[str, ...]:
    return tuple(sorted({k.split("/")[0] for k in _tables()}))


def _element_shells(basis: str, element: str, kind: str):
    t = _tables()
    key = f"{basis.strip().lower()}/{element}/{kind}"
    if key + "/l" not in t:
        raise KeyError(f"no {kind} shells for element {element!r} in basis {basis!r}")
    return t[key + "/l"], t[key + "/nprim"], t[key + "/exp"], t[key + "/coef"]


def pack_basis(atoms: list[tuple[str, np.ndarray]], basis: str, kind: str = "ao") -> BasisCartSoA:
    """Pack the AO (``kind='ao'``) or RICD aux (``kind='aux'``) basis of a molecule.

    Shells are laid out atom by atom in input order, each atom contributing its
    element's shells in table order -- the same order the reference's packer
    and RICD generator produce.
    """

    cxyz, pstart, nprim, ls, aostart, pexp, pcoef, satom = [], [], [], [], [], [], [], []
    prim_off = 0
    ao_off = 0
    for ia, (el, xyz) in enumerate(atoms):
        l, npr, e, c = _element_shells(basis, el, kind)
        xyz = np.asarray(xyz, dtype=np.float64).reshape(3)
        off = 0
        for s in range(l.size):
            n = int(npr[s])
            cxyz.append(xyz)
            pstart.append(prim_off)
            nprim.append(n)
            ls.append(int(l[s]))
            aostart.append(ao_off)
            satom.append(ia)
            pexp.append(e[off : off + n])
            pcoef.append(c[off : off + n])
            off += n
            prim_off += n
            ao_off += ncart(int(l[s]))
    i32 = lambda v: np.asarray(v, dtype=np.int32)  # noqa: E731
    return BasisCartSoA(
        shell_cxyz=np.asarray(cxyz, dtype=np.float64).reshape((-1, 3)),
        shell_prim_start=i32(pstart),
        shell_nprim=i32(nprim),
        shell_l=i32(ls),
        shell_ao_start=i32(aostart),
        prim_exp=np.concatenate(pexp) if pexp else np.zeros(0),
        prim_coef=np.concatenate(pcoef) if pcoef else np.zeros(0),
        shell_atom=i32(satom),
    )


def build_shell_pairs_l_order(basis: BasisCartSoA) -> ShellPairs:
    """Shell pairs (i >= j) in the reference's enumeration order, oriented l(A) >= l(B).

    Follows ``asuka/cueri/shell_pairs.py:72-115``: pairs are enumerated as
    ``for i: for j <= i``, and swapped when ``l(i) < l(j)``.
    """

    l = np.asarray(basis.shell_l, dtype=np.int32)
    npr = np.asarray(basis.shell_nprim, dtype=np.int32)
    n = l.size
    ii, jj = np.tril_indices(n)
    # np.tril_indices enumerates row-major: (0,0),(1,0),(1,1),(2,0),... == for i: for j<=i
    swap = l[ii] < l[jj]
    A = np.where(swap, jj, ii).astype(np.int32)
    B = np.where(swap, ii, jj).astype(np.int32)
    npair = (npr[A] * npr[B]).astype(np.int32)
    start = np.zeros(A.size + 1, dtype=np.int32)
    np.cumsum(npair, out=start[1:])
    return ShellPairs(sp_A=A, sp_B=B, sp_npair=npair, sp_pair_start=start)


def shell_to_atom_map(basis: BasisCartSoA, atom_coords_bohr: np.ndarray, tol: float = 1e-10) -> np.ndarray:
    """Owning atom of every shell, matched by centre (``asuka/integrals/int1e_cart.py:44``)."""

    if basis.shell_atom is not None:
        return np.asarray(basis.shell_atom, dtype=np.int32)
    R = np.asarray(atom_coords_bohr, dtype=np.float64).reshape((-1, 3))
    d2 = ((basis.shell_cxyz[:, None, :] - R[None, :, :]) ** 2).sum(-1)
    ia = np.argmin(d2, axis=1)
    if np.any(d2[np.arange(ia.size), ia] > tol * tol):
        raise ValueError(f"shell center does not match any atom within tol={tol:g}")
    return ia.astype(np.int32)


def with_coords(basis: BasisCartSoA, atom_coords_bohr: np.ndarray) -> BasisCartSoA:
    """Same basis with shell centres moved to new atom positions."""

    if basis.shell_atom is None:
        raise ValueError("basis has no shell->atom map")
    R = np.asarray(atom_coords_bohr, dtype=np.float64).reshape((-1, 3))
    return BasisCartSoA(
        shell_cxyz=np.ascontiguousarray(R[basis.shell_atom]),
        shell_prim_start=basis.shell_prim_start,
        shell_nprim=basis.shell_nprim,
        shell_l=basis.shell_l,
        shell_ao_start=basis.shell_ao_start,
        prim_exp=basis.prim_exp,
        prim_coef=basis.prim_coef,
        shell_atom=basis.shell_atom,
    )


def from_reference_like(obj, shell_atom: np.ndarray | None = None) -> BasisCartSoA:
    """Wrap any object exposing the reference ``BasisCartSoA`` fields."""

    return BasisCartSoA(
        shell_cxyz=np.ascontiguousarray(np.asarray(obj.shell_cxyz, dtype=np.float64)),
        shell_prim_start=np.ascontiguousarray(np.asarray(obj.shell_prim_start, dtype=np.int32)),
        shell_nprim=np.ascontiguousarray(np.asarray(obj.shell_nprim, dtype=np.int32)),
        shell_l=np.ascontiguousarray(np.asarray(obj.shell_l, dtype=np.int32)),
        shell_ao_start=np.ascontiguousarray(np.asarray(obj.shell_ao_start, dtype=np.int32)),
        prim_exp=np.ascontiguousarray(np.asarray(obj.prim_exp, dtype=np.float64)),
        prim_coef=np.ascontiguousarray(np.asarray(obj.prim_coef, dtype=np.float64)),
        shell_atom=None if shell_atom is None else np.asarray(shell_atom, dtype=np.int32),
    )
