"""Phase breakdown of one DF J/K + gradient step, and a driver for ncu captures.

    python -m asuka_b200.profile_step [--workload w8|decane|n2] [--steps N] [--precision fp64|mixed]
    python -m asuka_b200.profile_step --only deriv3c --steps 1     # one phase, for `ncu -k ...`

Uses an orthonormal random occupied block (the step's cost does not depend on
the density's values), so the launch list holds the step's kernels only.
"""

from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import basis as bm
from . import geometry as geo
from .df import DFEngine, cholesky_metric
from .grad import df_adjoints, df_contract

WORKLOADS = {
    "w8": lambda: geo.water_cluster(8, 0, "ma-tzvp"),
    "decane": lambda: geo.decane(0, "ma-svp"),
    "n2": lambda: geo.n2("ma-svp"),
    "w1": lambda: geo.water("ma-tzvp"),
    "w32": lambda: geo.water_cluster(32, 0, "ma-tzvp"),
    "w64": lambda: geo.water_cluster(64, 0, "ma-tzvp"),
    "w4q": lambda: geo.water_cluster(4, 0, "ma-qzvp"),
}


def setup(name: str):
    mol = WORKLOADS[name]()
    atoms = list(mol.atoms_bohr)
    ao = bm.pack_basis(atoms, mol.basis, "ao")
    aux = bm.pack_basis(atoms, mol.basis, "aux")
    eng = DFEngine(ao, aux)
    rng = np.random.default_rng(0)
    nocc = mol.nelectron // 2
    Cw = torch.as_tensor(np.linalg.qr(rng.standard_normal((ao.nao, nocc)))[0] * np.sqrt(2.0), device="cuda")
    R = torch.as_tensor(mol.coords_bohr, device="cuda")
    return mol, eng, Cw, R


def phases(eng: DFEngine, Cw: torch.Tensor, R: torch.Tensor, precision: str, X: torch.Tensor) -> dict:
    ev = {}

    def mark(k):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        ev[k] = e

    mark("start")
    eng.set_coords(R)
    mark("pair_tables")
    V = eng.metric()
    mark("metric")
    L = cholesky_metric(V)
    mark("cholesky")
    eng.int3c("Qmn", out=X, precision=precision)
    mark("int3c")
    E, J, K, saved = df_contract(eng, Cw, X, L, precision, mark)
    G3, G2 = df_adjoints(eng, Cw, saved, precision)
    mark("adjoints")
    grad = torch.zeros((eng.natm, 3), dtype=torch.float64, device="cuda")
    eng.deriv3c(G3, grad, precision=precision)
    mark("deriv3c")
    eng.deriv2c(G2, grad, precision=precision)
    mark("deriv2c")
    torch.cuda.synchronize()
    keys = list(ev)
    out = {k: ev[keys[i - 1]].elapsed_time(ev[k]) for i, k in enumerate(keys) if i > 0}
    out["total"] = ev["start"].elapsed_time(ev[keys[-1]])
    return out


def class_times(eng, mol, top: int = 20, precision: str = "fp64") -> dict:
    """Per-class device time of the 3c integrals and the 3c derivative contraction."""
    import ctypes
    import os
    import sys

    from . import _lib

    pc = 0 if precision == "fp64" else 1  # DFB_PREC_FP64 / DFB_PREC_MIXED for every class

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc"))
    import gen_classes

    nao = eng.nao
    X = torch.empty((eng.naux, nao, nao), dtype=torch.float64, device="cuda")
    X.fill_(1e-3)
    g = torch.zeros((eng.natm, 3), dtype=torch.float64, device="cuda")
    st = int(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    out = {}
    for deriv in (False, True):
        scr = eng._scratch_for(deriv)
        res = []
        for la, lb, lc, pairs, auxs in eng.classes3c:
            args = [la, lb, lc, ctypes.byref(eng.ps_ao), ctypes.byref(eng.axs), _lib.ptr(pairs), _lib.ptr(auxs),
                    pairs.numel() * auxs.numel(), -pairs.numel(), 0, pc, _lib.ptr(X), nao * nao,
                    nao, 1]
            fn = L.dfb_rys_deriv_prec if deriv else L.dfb_rys_int_prec
            if deriv:
                args += [_lib.ptr(g), eng.natm]
            args += [_lib.ptr(scr), scr.numel(), st]
            fn(*args)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(3):
                _lib.check(fn(*args), "class timing")
            e1.record()
            torch.cuda.synchronize()
            plan = (gen_classes.plan(la, lb, lc, deriv, f32=precision != "fp64")
                    if la <= gen_classes.LA_MAX and lc <= gen_classes.LC_MAX else None)
            res.append((e0.elapsed_time(e1) / 3, f"({la},{lb},{lc})", pairs.numel() * auxs.numel(),
                        "warp" if plan is None else f"thread FS={plan[0]}{' split' if plan[1] else ''}"))
        res.sort(reverse=True)
        key = "deriv3c" if deriv else "int3c"
        out[key] = {"total_ms": round(sum(r[0] for r in res), 3),
                    "warp_ms": round(sum(r[0] for r in res if r[3] == "warp"), 3),
                    "top": [[round(r[0], 3), r[1], r[2], r[3]] for r in res[:top]]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="w8", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "mixed_all"])
    ap.add_argument("--only", default=None, choices=[None, "int3c", "deriv3c", "metric", "deriv2c", "step"])
    ap.add_argument("--classes", action="store_true", help="time every angular class of int3c and deriv3c")
    ap.add_argument("--cls", default=None, metavar="LA,LB,LC",
                    help="keep only this 3c angular class (with --only int3c/deriv3c or --classes)")
    ap.add_argument("--streamed", type=int, default=0, metavar="NAUX_BLOCK",
                    help="streamed energy+gradient (3c recomputed per aux block of this size); prints peak HBM")
    args = ap.parse_args()
    mol, eng, Cw, R = setup(args.workload)
    if args.cls:
        want = tuple(int(v) for v in args.cls.split(","))
        eng.classes3c = [c for c in eng.classes3c if tuple(c[:3]) == want]
        if not eng.classes3c:
            raise SystemExit(f"class {want} does not occur in {args.workload}")
    if args.streamed:
        from .grad import df_energy_grad_streamed

        for i in range(max(1, args.steps)):
            st = {}
            E, g, _ = df_energy_grad_streamed(eng, Cw, aux_block=args.streamed, precision=args.precision, stats=st)
            print(json.dumps({"workload": args.workload, "nao": eng.nao, "naux": eng.naux, "nocc": Cw.shape[1],
                              "precision": args.precision, "run": i, "E2": float(E),
                              "grad_norm": float(g.norm()), "n_dropped_pairs": int(eng.n_dropped_pairs),
                              **{k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()}}))
        return
    if args.classes:
        print(json.dumps(class_times(eng, mol, precision=args.precision)))
        return
    X = torch.empty((eng.naux, eng.nao, eng.nao), dtype=torch.float64, device="cuda")
    if args.only in ("int3c", "deriv3c", "metric", "deriv2c"):
        g = torch.zeros((eng.natm, 3), dtype=torch.float64, device="cuda")
        bar2 = torch.ones((eng.naux, eng.naux), dtype=torch.float64, device="cuda")
        if args.only == "deriv3c":
            X.fill_(1e-3)
        for _ in range(args.steps):
            if args.only == "int3c":
                eng.int3c("Qmn", out=X, precision=args.precision)
            elif args.only == "metric":
                eng.metric()
            elif args.only == "deriv3c":
                eng.deriv3c(X, g, precision=args.precision)
            else:
                eng.deriv2c(bar2, g, precision=args.precision)
        torch.cuda.synchronize()
        print(json.dumps({"only": args.only, "steps": args.steps}))
        return
    phases(eng, Cw, R, args.precision, X)  # warm-up
    res = [phases(eng, Cw, R, args.precision, X) for _ in range(args.steps)]
    # median over steps: a step whose host side fell behind the device (page faults, the
    # allocator, Python) would otherwise inflate the phase it happened in
    avg = {k: float(np.median([r[k] for r in res])) for k in res[0]}
    print(json.dumps({"workload": args.workload, "nao": eng.nao, "naux": eng.naux, "precision": args.precision,
                      "ms": {k: round(v, 3) for k, v in avg.items()}}))


if __name__ == "__main__":
    main()
