"""Per-class precision autotuner for the mixed mode.

The FP32-component Rys kernels (``DFB_PREC_MIXED``) are faster than the FP64 ones but add
about 1e-7 relative error per integral; summed over a whole molecule that error reaches the
1e-6 Eh / 1e-6 Eh/bohr accuracy contract of the mixed step if every class runs in FP32.  This
tool measures, on the GPU, every angular class's contribution separately: one J/K + gradient
step with only that class's 3c integrals (or 3c derivative, or 2c derivative) in FP32, against
the all-FP64 step at the same density -- the first-order energy and gradient change the class
causes -- and the class's FP64 and FP32 kernel times.  It then admits classes greedily by
time saved per unit of error until the summed absolute energy change or any summed absolute
gradient component reaches its budget (a quarter of the contract by default), and writes the
admitted classes to ``asuka_b200/data/class_precision.json`` (read by
``asuka_b200.df.mixed_class_table``).

    python -m asuka_b200.tune_precision [--workload w8] [--e-budget 2.5e-7] [--g-budget 2.5e-7]

The reference has no counterpart: its mixed mode is all-or-nothing per kernel family
(``asuka/integrals/cueri_df.py:61-65``).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

import numpy as np
import torch

from . import _lib
from . import df as dfmod
from .grad import df_backward, df_forward
from .profile_step import WORKLOADS

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "class_precision.json")


def _density(mol, eng):
    """Converged FP64 RHF occupied block Cw of the workload (stored-B SCF)."""
    from .df import cholesky_metric, whiten_3c2e
    from .int1e import build_int1e
    from .scf import rhf_df

    int1e = build_int1e(eng.ao, mol.coords_bohr, mol.charges)
    L = cholesky_metric(eng.metric())
    B = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn")
    res = rhf_df(int1e.S, int1e.hcore, B, nelec=mol.nelectron, enuc=mol.energy_nuc())
    del B
    torch.cuda.empty_cache()
    nocc = mol.nelectron // 2
    return (res.mo_coeff[:, :nocc] * 2.0**0.5).contiguous(), res.e_tot


def _step(eng, Cw, R, X, precision):
    eng.set_coords(R)
    E, _J, _K, saved = df_forward(eng, Cw, precision, X=X, with_adjoints=True)
    g = df_backward(eng, Cw, saved, precision=precision)
    return float(E), g.cpu().numpy()


def _class_time(fn, args, reps=3) -> float:
    _lib.check(fn(*args), "class timing")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        _lib.check(fn(*args), "class timing")
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def measure(workload: str = "w8") -> dict:
    mol = WORKLOADS[workload]()
    from . import basis as bm

    atoms = list(mol.atoms_bohr)
    ao = bm.pack_basis(atoms, mol.basis, "ao")
    aux = bm.pack_basis(atoms, mol.basis, "aux")
    eng = dfmod.DFEngine(ao, aux)
    Cw, e_scf = _density(mol, eng)
    R = torch.as_tensor(mol.coords_bohr, dtype=torch.float64, device=eng.device)
    X = torch.empty((eng.naux, eng.nao, eng.nao), dtype=torch.float64, device=eng.device)
    E64, g64 = _step(eng, Cw, R, X, "fp64")
    Eall, gall = _step(eng, Cw, R, X, "mixed_all")
    rows = []
    kinds = [("int3c", (la, lb, lc)) for la, lb, lc, _p, _a in eng.classes3c]
    kinds += [("deriv3c", (la, lb, lc)) for la, lb, lc, _p, _a in eng.classes3c]
    kinds += [("deriv2c", (lp, 0, lq)) for lp, lq, _P, _Q in eng.classes2c]
    L = _lib.lib()
    st = int(torch.cuda.current_stream().cuda_stream)
    nao, naux = eng.nao, eng.naux
    gbuf = torch.zeros((eng.natm, 3), dtype=torch.float64, device=eng.device)
    bar2 = torch.full((naux, naux), 1e-3, dtype=torch.float64, device=eng.device)
    Xt = torch.full((naux, nao, nao), 1e-3, dtype=torch.float64, device=eng.device)
    t0 = time.time()
    try:
        for kind, cls in kinds:
            # the step with only this class in FP32
            table = {"int3c": set(), "deriv3c": set(), "deriv2c": set()}
            table[kind].add(cls)
            orig = dfmod.mixed_class_table
            dfmod.mixed_class_table = lambda _t=table: _t  # type: ignore[assignment]
            try:
                Ec, gc = _step(eng, Cw, R, X, "mixed")
            finally:
                dfmod.mixed_class_table = orig  # type: ignore[assignment]
            # kernel times, FP64 and FP32
            la, lb, lc = cls
            times = []
            for prec in (dfmod.PREC_FP64, dfmod.PREC_MIXED):
                if kind == "deriv2c":
                    P, Q = next((P, Q) for lp, lq, P, Q in eng.classes2c if (lp, 0, lq) == cls)
                    args = [la, 0, lc, ctypes.byref(eng.ps_aux), ctypes.byref(eng.axs), _lib.ptr(P), _lib.ptr(Q),
                            P.numel(), 0, 1, prec, _lib.ptr(bar2), naux, 1, 0, _lib.ptr(gbuf), eng.natm]
                    scr = eng._scratch_for(True)
                    fn = L.dfb_rys_deriv_prec
                else:
                    pairs, auxs = next((p, a) for a_, b_, c_, p, a in eng.classes3c if (a_, b_, c_) == cls)
                    args = [la, lb, lc, ctypes.byref(eng.ps_ao), ctypes.byref(eng.axs), _lib.ptr(pairs),
                            _lib.ptr(auxs), pairs.numel() * auxs.numel(), -pairs.numel(), 0, prec, _lib.ptr(Xt),
                            nao * nao, nao, 1]
                    if kind == "deriv3c":
                        args += [_lib.ptr(gbuf), eng.natm]
                        fn = L.dfb_rys_deriv_prec
                    else:
                        fn = L.dfb_rys_int_prec
                    scr = eng._scratch_for(kind == "deriv3c")
                times.append(_class_time(fn, args + [_lib.ptr(scr), scr.numel(), st]))
            dg = gc - g64
            rows.append({"kind": kind, "cls": list(cls), "dE": Ec - E64, "dg": dg.tolist(),
                         "dg_max": float(np.abs(dg).max()), "ms_fp64": times[0], "ms_fp32": times[1]})
    finally:
        dfmod.mixed_class_table.cache_clear()
    return {"workload": workload, "nao": nao, "naux": naux, "natm": eng.natm, "e_scf": e_scf, "E64": E64,
            "dE_all_mixed": Eall - E64, "dg_all_mixed": float(np.abs(gall - g64).max()), "rows": rows,
            "seconds": time.time() - t0}


def select(data: dict, e_budget: float, g_budget: float) -> dict:
    """Greedy admission by time saved per unit of (budget-normalised) error."""
    natm = data["natm"]
    cand = []
    for r in data["rows"]:
        gain = r["ms_fp64"] - r["ms_fp32"]
        if gain <= 0:
            continue
        cost = max(abs(r["dE"]) / e_budget, r["dg_max"] / g_budget, 1e-12)
        cand.append((gain / cost, r))
    cand.sort(key=lambda t: -t[0])
    e_sum = 0.0
    g_sum = np.zeros((natm, 3))
    chosen = {"int3c": [], "deriv3c": [], "deriv2c": []}
    saved = 0.0
    for _score, r in cand:
        e_new = e_sum + abs(r["dE"])
        g_new = g_sum + np.abs(np.asarray(r["dg"]))
        if e_new <= e_budget and float(g_new.max()) <= g_budget:
            e_sum, g_sum = e_new, g_new
            chosen[r["kind"]].append(r["cls"])
            saved += r["ms_fp64"] - r["ms_fp32"]
    return {"int3c": sorted(chosen["int3c"]), "deriv3c": sorted(chosen["deriv3c"]),
            "deriv2c": sorted(chosen["deriv2c"]), "bound_abs_dE": e_sum, "bound_max_abs_dg": float(g_sum.max()),
            "class_ms_saved": saved, "e_budget": e_budget, "g_budget": g_budget}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="w8", choices=sorted(WORKLOADS))
    ap.add_argument("--e-budget", type=float, default=2.5e-7)
    ap.add_argument("--g-budget", type=float, default=2.5e-7)
    ap.add_argument("--raw", default=None, help="also write the per-class measurements here (JSON)")
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args()
    data = measure(args.workload)
    if args.raw:
        with open(args.raw, "w") as f:
            json.dump(data, f)
    sel = select(data, args.e_budget, args.g_budget)
    sel.update(workload=args.workload, device=torch.cuda.get_device_name(),
               dE_all_mixed=data["dE_all_mixed"], dg_all_mixed=data["dg_all_mixed"])
    with open(args.out, "w") as f:
        json.dump(sel, f, indent=1)
    print(json.dumps({k: v for k, v in sel.items() if k not in ("int3c", "deriv3c", "deriv2c")}))
    print(json.dumps({k: len(sel[k]) for k in ("int3c", "deriv3c", "deriv2c")}))


if __name__ == "__main__":
    main()
