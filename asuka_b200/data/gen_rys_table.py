"""Generate ``rys_table.npz``: piecewise-Chebyshev Rys roots and weights.

The Rys quadrature of order ``n`` at argument ``T`` has nodes ``x_i`` in
(0, 1) (in the variable x = t^2) and weights ``w_i`` such that, for every
polynomial ``f`` of degree < 2n,

    int_0^1 f(t^2) exp(-T t^2) dt = sum_i w_i f(x_i),   sum_i w_i = F_0(T).

The reference evaluates them per call from the Boys moments F_m(T) with a
monomial Stieltjes procedure and a QL eigensolve
(``asuka/cueri/_eri_rys_cpu.pyx:547-672``), which loses accuracy quickly with
``n`` in double precision.  Here the same nodes and weights are computed once
in 100-digit arithmetic (mpmath): moments F_m(T) = 1F1(m+1/2; m+3/2; -T)/(2m+1),
Jacobi matrix by the Chebyshev algorithm on the moments, eigen-decomposition
(Golub-Welsch).  Each node/weight is then fitted on T in [0, T_MAX) by a
degree-``DEG`` Chebyshev interpolant per interval of width T_MAX/NINT, stored in the power
basis of the local variable u = 2(T - T0)/h - 1 for Horner evaluation.

For T >= T_MAX the Gauss-Hermite limit is exact to the working precision:
x_i = s_i^2 / T, w_i = W_i / sqrt(T), with s_i > 0 the positive roots of
H_{2n} and W_i their Gauss-Hermite weights; the neglected tail is O(exp(-T)).
Those ``s_i^2`` and ``W_i`` are stored too.

Output layout (float64):
    coef[n]  : (NINT, 2n, DEG+1)   rows 0..n-1 nodes, n..2n-1 weights
    herm[n]  : (2, n)              s_i^2 and W_i
"""

from __future__ import annotations

import multiprocessing as mproc
import os
import sys

import mpmath as mp
import numpy as np

NMAX = 10
T_MAX = 96.0
NINT = 192         # intervals of width 0.5 on [0, T_MAX)
DEG = 9
DPS = 110


def _boys(m: int, T):
    if T == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -T) / (2 * m + 1)


def rys_mp(n: int, T) -> tuple[list, list]:
    """High-precision Rys nodes/weights (ascending nodes)."""
    mp.mp.dps = DPS
    T = mp.mpf(T)
    mom = [_boys(k, T) for k in range(2 * n)]
    # Chebyshev algorithm (Gautschi) on ordinary moments -> recurrence coefficients.
    sig_prev = [mp.mpf(0)] * (2 * n)
    sig = list(mom)
    alpha = [mom[1] / mom[0]]
    beta = [mom[0]]
    for k in range(1, n):
        sig_new = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            sig_new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha.append(sig_new[k + 1] / sig_new[k] - sig[k] / sig[k - 1])
        beta.append(sig_new[k] / sig[k - 1])
        sig_prev, sig = sig, sig_new
    J = mp.matrix(n, n)
    for i in range(n):
        J[i, i] = alpha[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(beta[i + 1])
    E, Q = mp.eigsy(J)
    idx = sorted(range(n), key=lambda i: E[i])
    x = [E[i] for i in idx]
    w = [mom[0] * Q[0, i] ** 2 for i in idx]
    return x, w


def _hermite_limit(n: int):
    mp.mp.dps = DPS
    # Positive roots of H_{2n} and Gauss-Hermite weights via the Golub-Welsch
    # matrix of the (physicists') Hermite recurrence.
    m = 2 * n
    J = mp.matrix(m, m)
    for i in range(m - 1):
        J[i, i + 1] = J[i + 1, i] = mp.sqrt(mp.mpf(i + 1) / 2)
    E, Q = mp.eigsy(J)
    pairs = sorted((E[i], mp.sqrt(mp.pi) * Q[0, i] ** 2) for i in range(m))
    pos = [(s, W) for s, W in pairs if s > 0]
    return [float(s * s) for s, _ in pos], [float(W) for _, W in pos]


def _fit_interval(args):
    n, k = args
    mp.mp.dps = DPS
    t0 = mp.mpf(k) * (mp.mpf(T_MAX) / NINT)
    h = mp.mpf(T_MAX) / NINT
    npts = DEG + 1
    us = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / npts) for j in range(npts)]
    vals = []
    for u in us:
        x, w = rys_mp(n, t0 + (u + 1) * h / 2)
        vals.append(x + w)
    vals = np.array([[float(v) for v in row] for row in vals])  # (npts, 2n)
    # Chebyshev coefficients by the discrete cosine sums, then power basis.
    us_f = np.array([float(u) for u in us])
    V = np.polynomial.chebyshev.chebvander(us_f, DEG)  # (npts, DEG+1)
    cheb = np.linalg.solve(V, vals)  # (DEG+1, 2n)
    out = np.zeros((2 * n, DEG + 1))
    for i in range(2 * n):
        pw = np.polynomial.chebyshev.cheb2poly(cheb[:, i])
        out[i, : pw.size] = pw
    return n, k, out


def evaluate(table: dict, n: int, T: float) -> tuple[np.ndarray, np.ndarray]:
    """Evaluate a generated table the way the kernels do (Horner in u)."""
    if T >= T_MAX:
        s2, W = table[f"herm{n}"]
        return s2 / T, W / np.sqrt(T)
    h = T_MAX / NINT
    k = min(int(T / h), NINT - 1)
    u = 2.0 * (T - k * h) / h - 1.0
    c = table[f"coef{n}"][k]
    acc = c[:, DEG].copy()
    for d in range(DEG - 1, -1, -1):
        acc = acc * u + c[:, d]
    return acc[:n], acc[n:]


def main(out_path: str) -> None:
    jobs = [(n, k) for n in range(1, NMAX + 1) for k in range(NINT)]
    ctx = mproc.get_context("spawn")
    with ctx.Pool(max(1, os.cpu_count() or 1)) as pool:
        res = pool.map(_fit_interval, jobs, chunksize=4)
    table: dict[str, np.ndarray] = {}
    for n in range(1, NMAX + 1):
        table[f"coef{n}"] = np.zeros((NINT, 2 * n, DEG + 1))
        s2, W = _hermite_limit(n)
        table[f"herm{n}"] = np.array([s2, W])
    for n, k, out in res:
        table[f"coef{n}"][k] = out
    table["meta"] = np.array([NMAX, T_MAX, NINT, DEG], dtype=np.float64)
    np.savez_compressed(out_path, **table)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(here, "rys_table.npz"))
