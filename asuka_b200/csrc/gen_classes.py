"""Generate the class-specialised Rys kernel instantiations (dfb_cls_*.cu).

For every angular class (la >= lb, lc), both variants (integrals, derivative
contraction) and both component types (FP64, and the mixed-precision float
tables/accumulators) this picks the smallest split FS of the aux shell's
Cartesian components such that one thread's accumulators fit the register
budget, and emits an instantiation of ``k_rys_thread<LA, LB, LC, FS, DERIV, ...>``
with a dispatcher.  Classes that do not fit stay on the generic warp kernel.
One output file per (variant, type, la, lb) so the files compile in parallel.

    python asuka_b200/csrc/gen_classes.py
"""

from __future__ import annotations

import os

HERE = os.path.dirname(os.path.abspath(__file__))
LA_MAX = 3   # AO shells up to f
LC_MAX = 6   # aux shells up to i
FS_MAX = 28
ACC_BUDGET = {False: 40, True: 40}   # doubles of live accumulators per thread
G_BUDGET = 48                          # doubles of the three 2D recurrence tables (column-limited)


def ncart(l):
    return (l + 1) * (l + 2) // 2


def ncb(L):
    return L * (L + 1) * (L + 2) // 6


def comps(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def g_cost(nm, lc, nfs):
    """Largest column-limited recurrence-table size over the subsets of a split."""
    cs = comps(lc)
    worst = 0
    for f0 in range(0, len(cs), nfs):
        sub = cs[f0:f0 + nfs]
        worst = max(worst, (nm + 1) * sum(max(c[d] for c in sub) + 1 for d in range(3)))
    return worst


def nrange(lo, hi):
    return ncb(hi + 1) - ncb(lo) if hi >= lo else 0


def acc_per_f(la, lb, mode):
    """Accumulator doubles per aux component for the kernel modes of dfb_rys_tmpl.cuh."""
    if mode == 0:
        return nrange(la, la + lb)
    if mode == 1:
        return nrange(max(la - 1, 0), la + lb - 1) + nrange(la + 1, la + lb + 1) + nrange(la, la + lb + 1)
    if mode == 2:
        return (nrange(la - 1, la + lb - 1) if la > 0 else 0) + nrange(la + 1, la + lb + 1)
    return nrange(la, la + lb - 1) + nrange(la, la + lb + 1)


def _key(la, lb, lc, deriv):
    return f"{'d' if deriv else 'i'}{la}{lb}{lc}"


def plan(la, lb, lc, deriv, budget=None, f32=False):
    """(FS, SPLIT) for a class, or None when it stays on the generic warp kernel.

    ``budget`` overrides the accumulator budget.  Otherwise, for the FP64 kernels, the
    environment variable DFB_GEN_ACC_BUDGET_DERIV (derivative classes) or
    DFB_GEN_ACC_BUDGET_INT (integral classes) sets the budget of every class of that kind (the
    tuner's variant builds), else the measured per-class table (``class_tuning.json``,
    "acc_budget"), else ACC_BUDGET.  Budgets count the live accumulators (the ones the
    epilogue reads) in doubles.  The mixed-precision kernels (``f32``) hold float accumulators
    and recurrence tables, so the same registers hold twice as many elements; their budget
    counts floats: DFB_GEN_ACC_BUDGET_DERIV_F32 / DFB_GEN_ACC_BUDGET_INT_F32 (variant builds),
    else the table's "acc_budget_f32", else twice the FP64 class's budget.
    """
    gbudget = 2 * G_BUDGET if f32 else G_BUDGET
    if budget is None:
        kind = "DERIV" if deriv else "INT"
        env = os.environ.get(f"DFB_GEN_ACC_BUDGET_{kind}_F32" if f32 else f"DFB_GEN_ACC_BUDGET_{kind}")
        if env:
            budget = int(env)
        elif f32 and _key(la, lb, lc, deriv) in tuning("acc_budget_f32"):
            budget = tuning("acc_budget_f32")[_key(la, lb, lc, deriv)]
        else:
            budget = tuning("acc_budget").get(_key(la, lb, lc, deriv), ACC_BUDGET[deriv])
            if f32:
                budget *= 2
    elif f32:
        budget *= 2
    nm = la + lb + (1 if deriv else 0)
    nf = ncart(lc)
    modes = [(1, False), (None, True)] if deriv else [(0, False)]
    best = None
    for mode, split in modes:
        per_f = max(acc_per_f(la, lb, 2), acc_per_f(la, lb, 3)) if split else acc_per_f(la, lb, mode)
        for fs in range(1, min(nf, FS_MAX) + 1):
            nfs = -(-nf // fs)
            if -(-nf // nfs) != fs:
                continue  # keep the split exact (no empty subsets)
            if per_f * nfs <= budget and g_cost(nm, lc, nfs) <= gbudget:
                # each pass repeats the task's roots and recurrence tables: fewest passes wins,
                # the unsplit form on a tie
                passes = fs * (2 if split else 1)
                if best is None or passes < best[0]:
                    best = (passes, fs, split)
                break
    return None if best is None else (best[1], best[2])


STAGE_MAX_ROOTS = 3  # tables of at most 3 roots (92 KB) fit beside 2 register-limited blocks per SM


def staged(la, lb, lc, deriv, f32=False):
    """Whether the class kernel copies its Rys table into shared memory (k_rys_thread STAGE).

    DFB_GEN_STAGE=1 stages every eligible class (the tuner's variant build); otherwise the
    measured table decides ("stage" for the FP64 kernels, "stage_f32" for the FP32 ones).
    Eligible: at most STAGE_MAX_ROOTS Rys roots."""
    if (la + lb + lc + (1 if deriv else 0)) // 2 + 1 > STAGE_MAX_ROOTS:
        return False
    if os.environ.get("DFB_GEN_STAGE"):
        return os.environ["DFB_GEN_STAGE"] == "1"
    return bool(tuning("stage_f32" if f32 else "stage").get(_key(la, lb, lc, deriv), 0))


def tuning(field: str = "min_blocks") -> dict:
    """Per-class choices measured by asuka_b200.tune_classes ("min_blocks": launch bounds,
    "acc_budget": accumulator budget of the component split); empty when absent or when
    DFB_GEN_NO_TUNING is set (a build with every class at the default shape)."""
    import json

    p = os.path.join(HERE, "class_tuning.json")
    if os.environ.get("DFB_GEN_NO_TUNING") or not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f).get(field, {})


def _groups():
    """Files of the generated set: one per (variant, precision, la, lb) so they compile in parallel."""
    out = []
    for deriv in (False, True):
        for f32 in (False, True):
            for la in range(LA_MAX + 1):
                for lb in range(la + 1):
                    cls = [(la, lb, lc, *pl) for lc in range(LC_MAX + 1)
                           if (pl := plan(la, lb, lc, deriv, f32=f32)) is not None]
                    if cls:
                        out.append((f"dfb_cls_{'d' if deriv else 'i'}{'f' if f32 else ''}{la}{lb}", deriv, f32, la, lb,
                                    cls))
    return out


def _write(name: str, text: str) -> None:
    """Write a generated file only when its content changes (keeps the build incremental)."""
    path = os.path.join(HERE, name)
    if os.path.exists(path):
        with open(path) as f:
            if f.read() == text:
                return
    with open(path, "w") as f:
        f.write(text)


def main() -> None:
    tune = tuning()
    groups = _groups()
    keep = {name + ".cu" for name, *_ in groups}
    for old in os.listdir(HERE):
        if old.startswith("dfb_cls_") and old.endswith(".cu") and old not in keep:
            os.remove(os.path.join(HERE, old))
    for name, deriv, f32, la, lb, cls in groups:
        lines = [
            "// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.",
            '#include "dfb_rys_tmpl.cuh"',
            "",
            "namespace dfb {",
            f"int {name}_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {{",
        ]
        for (a, b, c, fs, split) in cls:
            minb = 1 if f32 else int(tune.get(_key(a, b, c, deriv), 1))
            stage = staged(a, b, c, deriv, f32)
            kern = (f"k_rys_thread<{a}, {b}, {c}, {fs}, {'true' if deriv else 'false'}, "
                    f"{'true' if split else 'false'}, {minb}, {'float' if f32 else 'double'}, "
                    f"{'true' if stage else 'false'}>")
            nr = (a + b + c + (1 if deriv else 0)) // 2 + 1
            lines.append(f"    if (lc == {c}) {{")
            if stage:  # the Rys table after the gradient buffer and the root slots
                lines.append(f"        const long ng = (long)(smem / sizeof(double)) - 256L * {nr};")
                lines.append(f"        const size_t sm = sizeof(double) * (size_t)(rys_stage_offset(ng, {nr}) + "
                             f"rys_stage_doubles(g.tab.nint, {nr}));")
                lines.append("        static size_t attr[64];")
                lines.append("        int dev = 0;")
                lines.append("        cudaGetDevice(&dev);")
                lines.append("        if (sm > attr[dev & 63]) {")
                lines.append(f"            cudaFuncSetAttribute({kern}, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);")
                lines.append("            attr[dev & 63] = sm;")
                lines.append("        }")
                lines.append(f"        {kern}<<<dim3((unsigned)nblk, {fs * (2 if split else 1)}), 128, sm, st>>>(g);")
            else:
                lines.append(f"        {kern}<<<dim3((unsigned)nblk, {fs * (2 if split else 1)}), 128, smem, st>>>(g);")
            lines.append("        return 1;")
            lines.append("    }")
        lines += ["    return 0;", "}", "}  // namespace dfb", ""]
        _write(name + ".cu", "\n".join(lines))
    # dispatcher header
    hdr = ["// Generated by gen_classes.py -- dispatch over the class-specialised kernels.", "#pragma once",
           '#include "dfb_rys_tmpl.cuh"', "", "namespace dfb {"]
    for name, *_ in groups:
        hdr.append(f"int {name}_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);")
    hdr += ["", "// f32: the mixed-precision variant (float recurrence tables and accumulators)",
            "inline int tmpl_launch(int la, int lb, int lc, bool deriv, bool f32, const TmplArgs& g, long nblk,",
            "                       size_t smem, cudaStream_t st) {"]
    for name, deriv, f32, la, lb, _cls in groups:
        hdr.append(f"    if ({'deriv' if deriv else '!deriv'} && {'f32' if f32 else '!f32'} && la == {la} && lb == {lb})"
                   f" return {name}_launch(lc, g, nblk, smem, st);")
    hdr += ["    return 0;", "}", ""]
    # host-side query: is a class served by a specialised kernel?
    hdr.append("inline bool tmpl_has(int la, int lb, int lc, bool deriv, bool f32) {")
    for deriv in (False, True):
        for f32 in (False, True):
            keys = [f"{{{la}, {lb}, {lc}}}" for la in range(LA_MAX + 1) for lb in range(la + 1)
                    for lc in range(LC_MAX + 1) if plan(la, lb, lc, deriv, f32=f32) is not None]
            hdr.append(f"    static const int k{'d' if deriv else 'i'}{'f' if f32 else ''}[][3] = {{{', '.join(keys)}}};")
    hdr += ["    const int (*k)[3] = deriv ? (f32 ? kdf : kd) : (f32 ? kif : ki);",
            "    const int n = deriv ? (f32 ? (int)(sizeof(kdf) / sizeof(kdf[0])) : (int)(sizeof(kd) / sizeof(kd[0])))",
            "                        : (f32 ? (int)(sizeof(kif) / sizeof(kif[0])) : (int)(sizeof(ki) / sizeof(ki[0])));",
            "    for (int i = 0; i < n; ++i)",
            "        if (k[i][0] == la && k[i][1] == lb && k[i][2] == lc) return true;",
            "    return false;", "}", "}  // namespace dfb", ""]
    _write("dfb_cls_dispatch.h", "\n".join(hdr))
    print("generated", len(groups), "groups")


if __name__ == "__main__":
    import sys

    if len(sys.argv) > 1:  # generate into another directory (the tuner's variant builds)
        HERE = os.path.abspath(sys.argv[1])
    main()
