"""Generate the class-specialised Rys kernel instantiations (dfb_cls_*.cu).

For every angular class (la >= lb, lc) and both variants (integrals,
derivative contraction) this picks the smallest split FS of the aux shell's
Cartesian components such that one thread's accumulators fit the register
budget, and emits an instantiation of ``k_rys_thread<LA, LB, LC, FS, DERIV>``
with a dispatcher.  Classes that do not fit stay on the generic warp kernel.
One output file per (variant, la) so the files compile in parallel.

    python asuka_b200/csrc/gen_classes.py
"""

from __future__ import annotations

import os

HERE = os.path.dirname(os.path.abspath(__file__))
LA_MAX = 3   # AO shells up to f
LC_MAX = 6   # aux shells up to i
FS_MAX = 16
ACC_BUDGET = {False: 36, True: 60}   # doubles of accumulators per thread
G_BUDGET = 48                          # doubles of the three 2D recurrence tables


def ncart(l):
    return (l + 1) * (l + 2) // 2


def ncb(L):
    return L * (L + 1) * (L + 2) // 6


def plan(la, lb, lc, deriv):
    nm = la + lb + (1 if deriv else 0)
    lmin = (la - 1 if la > 0 else 0) if deriv else la
    ne = ncb(nm + 1) - ncb(lmin)
    nf = ncart(lc)
    nw = 3 if deriv else 1
    if 3 * (nm + 1) * (lc + 1) > G_BUDGET:
        return None
    for fs in range(1, min(nf, FS_MAX) + 1):
        nfs = -(-nf // fs)
        if -(-nf // nfs) != fs:
            continue  # keep the split exact (no empty subsets)
        if nw * ne * nfs <= ACC_BUDGET[deriv]:
            return fs
    return None


def main() -> None:
    for old in os.listdir(HERE):
        if old.startswith("dfb_cls_") and old.endswith(".cu"):
            os.remove(os.path.join(HERE, old))
    groups = []
    for deriv in (False, True):
        for la in range(LA_MAX + 1):
            cls = []
            for lb in range(la + 1):
                for lc in range(LC_MAX + 1):
                    fs = plan(la, lb, lc, deriv)
                    if fs is not None:
                        cls.append((la, lb, lc, fs))
            if not cls:
                continue
            name = f"dfb_cls_{'d' if deriv else 'i'}{la}"
            groups.append(name)
            lines = [
                "// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.",
                '#include "dfb_rys_tmpl.cuh"',
                "",
                "namespace dfb {",
                f"int {name}_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {{",
                "    (void)la;",
            ]
            for (a, b, c, fs) in cls:
                kern = f"k_rys_thread<{a}, {b}, {c}, {fs}, {'true' if deriv else 'false'}>"
                lines.append(f"    if (lb == {b} && lc == {c}) {{")
                lines.append(f"        {kern}<<<dim3((unsigned)nblk, {fs}), 128, smem, st>>>(g);")
                lines.append("        return 1;")
                lines.append("    }")
            lines += ["    return 0;", "}", "}  // namespace dfb", ""]
            with open(os.path.join(HERE, name + ".cu"), "w") as f:
                f.write("\n".join(lines))
    # dispatcher header
    hdr = ["// Generated by gen_classes.py -- dispatch over the class-specialised kernels.", "#pragma once",
           '#include "dfb_rys_tmpl.cuh"', "", "namespace dfb {"]
    for name in groups:
        hdr.append(f"int {name}_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);")
    hdr += ["", "inline int tmpl_launch(int la, int lb, int lc, bool deriv, const TmplArgs& g, long nblk, size_t smem,",
            "                       cudaStream_t st) {"]
    for name in groups:
        d = name[8] == "d"
        la = int(name[9:])
        hdr.append(f"    if ({'deriv' if d else '!deriv'} && la == {la}) return {name}_launch(la, lb, lc, g, nblk, smem, st);")
    hdr += ["    return 0;", "}", "}  // namespace dfb", ""]
    with open(os.path.join(HERE, "dfb_cls_dispatch.h"), "w") as f:
        f.write("\n".join(hdr))
    print("generated", len(groups), "groups")


if __name__ == "__main__":
    main()
