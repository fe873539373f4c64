"""Cartesian -> real spherical AO transforms (the ``ao_rep='sph'`` seams).

``cart2sph_matrix(l)`` is the (ncart, 2l+1) matrix of the real solid harmonics
in the Cartesian monomials of one shell.  The convention is the one the reference
uses (``asuka/cueri/sph.py:95``, PySCF's with the 'sp' normalisation):
* l = 0 and l = 1 are the identity (p functions stay x, y, z);
* for l >= 2, the columns are m = -l..l, each sqrt((2l+1)/4pi) r^l Y_lm with
  cos(m phi) for m > 0, sin(|m| phi) for m < 0, and no Condon-Shortley phase;
* the rows follow this package's Cartesian order (x-major: for lx = l..0, ly = l-lx..0).

The coefficients are generated from the closed form of the real solid harmonics
(Helgaker, Jorgensen and Olsen, Molecular Electronic-Structure Theory, eqs. 6.4.47-6.4.50),
not tabulated, so any l up to the engine's maximum is available.

The AO-side transforms of the DF seams: X_sph[P] = T^T X_cart[P] T with T the
block-diagonal (nao_cart, nao_sph) matrix of the shells, and orbitals C_cart = T C_sph.
The aux basis stays Cartesian, as in the reference.
"""

from __future__ import annotations

from fractions import Fraction
from functools import lru_cache
from math import comb, factorial, pi, sqrt

import numpy as np
import torch

from .basis import ncart


def nsph(l: int) -> int:
    if l < 0:
        raise ValueError("l must be >= 0")
    return 2 * l + 1


def _cart_index(lx: int, ly: int, l: int) -> int:
    return ((l - lx) * (l - lx + 1)) // 2 + (l - lx - ly)


@lru_cache(maxsize=None)
def cart2sph_matrix(l: int) -> np.ndarray:
    """(ncart(l), 2l+1) Cartesian -> spherical coefficients (see module docstring)."""
    if l < 0:
        raise ValueError("l must be >= 0")
    if l <= 1:
        return np.eye(ncart(l))
    out = np.zeros((ncart(l), 2 * l + 1))
    for m in range(-l, l + 1):
        am = abs(m)
        # N_lm = sqrt(2 (l+|m|)! (l-|m|)! / 2^{delta_m0}) / (2^|m| l!)
        norm = sqrt(2.0 * factorial(l + am) * factorial(l - am) / (2.0 if m == 0 else 1.0)) / (2 ** am * factorial(l))
        # 2v runs over even values for m >= 0 and odd values for m < 0
        v2s = range(0, am + 1, 2) if m >= 0 else range(1, am + 1, 2)
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                for v2 in v2s:
                    sign = -1 if ((t + (v2 - (0 if m >= 0 else 1)) // 2) % 2) else 1
                    c = Fraction(sign) * Fraction(1, 4 ** t) * comb(l, t) * comb(l - t, am + t) * comb(t, u) * comb(am, v2)
                    lx = 2 * t + am - 2 * u - v2
                    ly = 2 * u + v2
                    lz = l - 2 * t - am
                    out[_cart_index(lx, ly, l), m + l] += float(c) * norm
    return out * sqrt((2 * l + 1) / (4 * pi))


def cart2sph_ao_matrix(shell_l, device=None) -> torch.Tensor:
    """Block-diagonal T (nao_cart, nao_sph) over the shells, in shell order."""
    ls = [int(l) for l in np.asarray(shell_l)]
    nc = sum(ncart(l) for l in ls)
    ns = sum(nsph(l) for l in ls)
    T = np.zeros((nc, ns))
    r = c = 0
    for l in ls:
        T[r:r + ncart(l), c:c + nsph(l)] = cart2sph_matrix(l)
        r += ncart(l)
        c += nsph(l)
    return torch.as_tensor(T, dtype=torch.float64, device=device)


def int3c_cart_to_sph(X: torch.Tensor, T: torch.Tensor, layout: str = "Qmn", q_block: int = 256) -> torch.Tensor:
    """X_sph[P] = T^T X_cart[P] T on the AO indices; returns a new tensor in the same layout."""
    if layout == "mnQ":
        return int3c_cart_to_sph(X.permute(2, 0, 1), T, "Qmn", q_block).permute(1, 2, 0).contiguous()
    if layout != "Qmn":
        raise ValueError("layout must be 'mnQ' or 'Qmn'")
    naux = X.shape[0]
    ns = T.shape[1]
    out = torch.empty((naux, ns, ns), dtype=torch.float64, device=X.device)
    for q0 in range(0, naux, q_block):
        q1 = min(naux, q0 + q_block)
        torch.matmul(T.T, torch.matmul(X[q0:q1], T), out=out[q0:q1])
    return out


def sph_coeff_sph_to_cart(C_sph, shell_l, device=None) -> torch.Tensor:
    """C_cart = T C_sph: spherical-AO orbitals in the Cartesian AO layout of the kernels
    (``asuka/integrals/cueri_df.py:586`` sph_coeff_sph_to_cart_device)."""
    C = torch.as_tensor(C_sph, dtype=torch.float64, device=device)
    T = cart2sph_ao_matrix(shell_l, device=C.device)
    if C.ndim != 2 or C.shape[0] != T.shape[1]:
        raise ValueError(f"C_sph must have shape ({T.shape[1]}, norb)")
    return T @ C
