"""Batched DF J/K builds for many molecules, replayed as one CUDA graph.

The workload is a set of independent molecules (seeded water clusters of
uneven size), each needing the DF Coulomb and exchange matrices for its own
occupied orbitals, the inner step of every molecule's SCF cycle
(``asuka/hf/df_jk_streamed.py:167-325`` for one molecule).  The geometry-fixed
work of every molecule (bases, screened pair lists, pair tables, metric and its
Cholesky factor, and for mixed precision the split L^-1) is done once at
set-up.  The J/K builds of all molecules are captured into ONE CUDA graph, so a
replay issues every class kernel, GEMM and solve of the batch with a single
launch from the host.

Per molecule, the integrals are computed in aux blocks into one shared block
buffer (sized by ``block_bytes``):

* pass 1, per block: X_b -> Y_b = X_b Cw, written into the shared Y buffer;
* rho from Y, d = V^-1 rho (two triangular solves), W = L^-1 Y in place,
  K = sum_Q W_Q W_Q^T by aux chunks;
* pass 2: J = sum_P d_P X_P.  When one block holds all of a molecule's aux
  functions, X is still in the buffer and the integrals are not recomputed;
  otherwise the blocks are recomputed (direct DF).

``precision='mixed'`` runs the exchange update K = W W^T as split-BF16 GEMMs
with FP32 accumulation (``asuka_b200.mixed``); with ``mixed_solve=True`` the
solve W = L^-1 Y also runs as a split-BF16 GEMM with a precomputed L^-1.  That
GEMM's error grows with the metric's condition number (about 1e-4 relative in
K for the ma-QZVP/RICD aux basis, against 1e-7 for the exchange update alone),
so it is off by default.  The integrals, the half-transform Y = X Cw and J stay
FP64.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import basis as bm
from . import geometry as geo
from . import linalg as _la
from . import mixed as _mixed
from . import tc as _tc
from .df import DFEngine, ScratchHolder, cholesky_metric


@dataclass
class _Member:
    eng: DFEngine
    L: torch.Tensor
    nocc: int
    max_naux: int        # aux functions per block
    single_block: bool   # X of all aux functions fits one block: no recompute in pass 2
    Cw: torch.Tensor     # static input (nao, nocc)
    J: torch.Tensor      # static outputs (nao, nao)
    K: torch.Tensor
    Linv_split: tuple | None = None
    Linv_blocks: list | None = None  # inverted diagonal blocks of L (block substitution)


def water_cluster_batch(nmol: int = 64, nmin: int = 1, nmax: int = 16, basis: str = "ma-qzvp"):
    """Molecule i: n_i ~ U{nmin..nmax} monomers from default_rng(i), then the seeded cluster of seed i."""
    mols = []
    for i in range(nmol):
        n = int(np.random.default_rng(i).integers(nmin, nmax + 1))
        mols.append(geo.water_cluster(n, i, basis))
    return mols


class BatchedDFJK:
    """J/K builds of a batch of closed-shell molecules, captured in one CUDA graph.

    ``run(Cws)`` takes one occupied-orbital block Cw = C_occ sqrt(occ) per molecule
    (host or device, (nao_i, nocc_i) FP64) and returns the list of (J_i, K_i), both
    symmetric (nao_i, nao_i) device tensors owned by the batch (overwritten by the next run).
    """

    def __init__(self, mols, precision: str = "fp64", block_bytes: int = 4 << 30, aux_block_min: int = 64,
                 device=None, graph: bool = True, mixed_solve: bool = False):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.mixed_solve = bool(mixed_solve) and precision == "mixed"
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.scratch = ScratchHolder()
        self.members: list[_Member] = []
        xb_need = y_need = 0
        for mol in mols:
            atoms = list(mol.atoms_bohr)
            ao = bm.pack_basis(atoms, mol.basis, "ao")
            aux = bm.pack_basis(atoms, mol.basis, "aux")
            eng = DFEngine(ao, aux, device=self.device, scratch=self.scratch)
            L = cholesky_metric(eng.metric())
            nao, naux = eng.nao, eng.naux
            nocc = mol.nelectron // 2
            per_aux = nao * nao * 8
            max_naux = max(aux_block_min, int(block_bytes // per_aux))
            blocks = eng.aux_blocks(max_naux)
            bmax = max(p1 - p0 for p0, p1, _ in blocks)
            xb_need = max(xb_need, bmax * nao * nao)
            y_need = max(y_need, naux * nao * nocc)
            m = _Member(eng, L, nocc, max_naux, len(blocks) == 1,
                        torch.zeros((nao, nocc), dtype=torch.float64, device=self.device),
                        torch.zeros((nao, nao), dtype=torch.float64, device=self.device),
                        torch.zeros((nao, nao), dtype=torch.float64, device=self.device))
            m.Linv_blocks = _la.diag_block_inverses(L)
            if self.mixed_solve:
                Linv = torch.linalg.solve_triangular(L, torch.eye(naux, dtype=L.dtype, device=L.device), upper=False)
                m.Linv_split = _mixed.split3(Linv)
                del Linv
            self.members.append(m)
        self.Xb = torch.zeros(max(xb_need, 1), dtype=torch.float64, device=self.device)
        self.Y = torch.zeros(max(y_need, 1), dtype=torch.float64, device=self.device)
        self.graph = None
        self._use_graph = graph
        self._pool = None

    # ---------------------------------------------------------------- one molecule
    def _jk_one(self, m: _Member) -> None:
        eng, L, Cw = m.eng, m.L, m.Cw
        nao, naux, nocc = eng.nao, eng.naux, m.nocc
        blocks = eng.aux_blocks(m.max_naux)
        bmax = max(p1 - p0 for p0, p1, _ in blocks)
        Xbuf = self.Xb[: bmax * nao * nao].view(bmax, nao, nao)
        if eng.n_dropped_pairs:
            Xbuf.zero_()  # screened-out pairs are never written; the buffer is shared by all molecules
        Y = self.Y[: naux * nao * nocc].view(naux, nao * nocc)
        mixed = self.precision == "mixed"
        for p0, p1, blk in blocks:
            Xb = eng.int3c_block(blk, p0, p1, out=Xbuf[: p1 - p0], dropped_zero=True)
            torch.matmul(Xb.view(-1, nao), Cw, out=Y[p0:p1].view(-1, nocc))
        rho = Y @ Cw.reshape(-1)
        t = torch.linalg.solve_triangular(L, rho.view(-1, 1), upper=False)
        d = torch.linalg.solve_triangular(L.T, t, upper=True).view(-1)
        if self.mixed_solve:
            ncol = max(nocc, ((1 << 28) // max(naux, 1)) // nocc * nocc)
            for c0 in range(0, nao * nocc, ncol):
                c1 = min(nao * nocc, c0 + ncol)
                Y[:, c0:c1] = _mixed.matmul(None, Y[:, c0:c1].contiguous(), kblock=4096, a_split=m.Linv_split)
        else:
            _la.solve_lower(L, Y, m.Linv_blocks, out=Y)
        W3 = Y.view(naux, nao, nocc)
        K = m.K
        K.zero_()
        qb = max(1, (1 << 27) // max(nao * nocc, 1))
        if mixed:
            _tc.syrk_qblocks(W3, out=K)  # split-BF16 tcgen05 update, W read in place
        for q0 in range(0, 0 if mixed else naux, qb):
            Wc = W3[q0:q0 + qb].permute(1, 0, 2).reshape(nao, -1)
            K.addmm_(Wc, Wc.T)
        K.copy_(0.5 * (K + K.T))
        J = m.J
        J.zero_()
        Jf = J.view(-1)
        for p0, p1, blk in blocks:
            if m.single_block:
                Xb = Xbuf[: p1 - p0]
            else:
                Xb = eng.int3c_block(blk, p0, p1, out=Xbuf[: p1 - p0], dropped_zero=True)
            Jf.addmv_(Xb.view(p1 - p0, -1).T, d[p0:p1])
        J.copy_(0.5 * (J + J.T))

    def _all(self) -> None:
        for m in self.members:
            self._jk_one(m)

    # ---------------------------------------------------------------- capture and replay
    def capture(self) -> None:
        """Run the batch once eagerly (allocates scratch, warms the libraries), then capture it."""
        self._all()
        torch.cuda.synchronize(self.device)
        if not self._use_graph:
            return
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="thread_local"):
            self._all()
        torch.cuda.synchronize(self.device)

    def set_orbitals(self, Cws) -> None:
        for m, Cw in zip(self.members, Cws):
            m.Cw.copy_(torch.as_tensor(Cw, dtype=torch.float64), non_blocking=True)

    def replay(self) -> None:
        if self.graph is None:
            self._all()
        else:
            self.graph.replay()

    def run(self, Cws):
        if len(Cws) != len(self.members):
            raise ValueError("one Cw per molecule is required")
        self.set_orbitals(Cws)
        if self.graph is None and self._use_graph:
            self.capture()
        self.replay()
        return [(m.J, m.K) for m in self.members]

    @property
    def sizes(self):
        return [(m.eng.nao, m.eng.naux, m.nocc, m.single_block) for m in self.members]


def main():
    """Time one graph replay of the batch (FP64 and/or mixed).

    python -m asuka_b200.batch [--nmol 64] [--nmin 1] [--nmax 16] [--basis ma-qzvp] [--precision fp64,mixed]
    """
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser()
    ap.add_argument("--nmol", type=int, default=64)
    ap.add_argument("--nmin", type=int, default=1)
    ap.add_argument("--nmax", type=int, default=16)
    ap.add_argument("--basis", default="ma-qzvp")
    ap.add_argument("--precision", default="fp64,mixed")
    ap.add_argument("--replays", type=int, default=2)
    ap.add_argument("--block-gb", type=float, default=4.0)
    ap.add_argument("--mixed-solve", action="store_true")
    args = ap.parse_args()
    mols = water_cluster_batch(args.nmol, args.nmin, args.nmax, args.basis)
    out = {"workload": f"{args.nmol} water clusters, n~U{{{args.nmin}..{args.nmax}}}, {args.basis} + RICD",
           "n_monomers": [m.natm // 3 for m in mols]}
    ref = None
    for prec in args.precision.split(","):
        torch.cuda.reset_peak_memory_stats()
        t0 = time.perf_counter()
        b = BatchedDFJK(mols, precision=prec, block_bytes=int(args.block_gb * (1 << 30)),
                        mixed_solve=args.mixed_solve)
        torch.cuda.synchronize()
        t_setup = time.perf_counter() - t0
        Cws = []
        rng = np.random.default_rng(0)  # the same orbitals for every precision
        for nao, naux, nocc, _ in b.sizes:
            Cws.append(torch.as_tensor(np.linalg.qr(rng.standard_normal((nao, nocc)))[0] * np.sqrt(2.0), device="cuda"))
        t0 = time.perf_counter()
        b.set_orbitals(Cws)
        b.capture()
        t_capture = time.perf_counter() - t0
        ms = []
        for _ in range(args.replays):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            b.replay()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        jk = [(J.clone(), K.clone()) for J, K in [(m.J, m.K) for m in b.members]]
        rec = {"setup_s": round(t_setup, 2), "eager_plus_capture_s": round(t_capture, 2),
               "replay_ms": [round(x, 1) for x in ms], "peak_hbm_bytes": int(torch.cuda.max_memory_allocated()),
               "nao_max": max(s[0] for s in b.sizes), "naux_max": max(s[1] for s in b.sizes),
               "sum_nao": sum(s[0] for s in b.sizes), "recomputed_molecules": sum(not s[3] for s in b.sizes)}
        if ref is None:
            ref = jk
        else:
            rec["max_rel_dK_vs_first"] = max(float((K - K0).abs().max() / K0.abs().max())
                                             for (J, K), (J0, K0) in zip(jk, ref))
            rec["max_rel_dJ_vs_first"] = max(float((J - J0).abs().max() / J0.abs().max())
                                             for (J, K), (J0, K0) in zip(jk, ref))
        out[prec] = rec
        del b
        torch.cuda.empty_cache()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
