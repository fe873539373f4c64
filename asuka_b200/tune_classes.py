"""Measured per-class launch bounds for the class-specialised Rys kernels.

The thread kernels run 128 threads per block.  By default the compiler may give a
thread up to 255 registers (the classes take 150-170, i.e. 3 resident blocks per SM);
capping them at 128 (4 blocks per SM) helps the classes whose working set still fits and
hurts the ones that then spill.  Which is which is measured, not guessed:

    python -m asuka_b200.tune_classes build                   # (no GPU) variant library, every class capped
    python -m asuka_b200.tune_classes measure w8 w4q --out T  # (GPU) time every class with both libraries
    cp T asuka_b200/csrc/class_tuning.json && python asuka_b200/csrc/gen_classes.py && python -m asuka_b200.build

A class gets the 4-block bound when it is at least ``MIN_GAIN`` faster with it on every
workload that contains it; ``gen_classes.py`` reads the table when generating the kernels.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
VARIANT = os.path.join(HERE, "_tune", "libdfb_minb4.so")
MIN_GAIN = 0.03


def _times(workload: str, lib: str | None) -> dict:
    env = dict(os.environ)
    env.pop("DFB_LIB_PATH", None)
    if lib:
        env["DFB_LIB_PATH"] = lib
    code = ("import json; from asuka_b200.profile_step import setup, class_times; "
            f"mol, eng, Cw, R = setup({workload!r}); print(json.dumps(class_times(eng, mol, top=10000)))")
    out = subprocess.run([sys.executable, "-c", code], env=env, check=True, capture_output=True, text=True,
                         cwd=os.path.dirname(HERE)).stdout
    res = json.loads(out.strip().splitlines()[-1])
    return {("d" if k == "deriv3c" else "i") + c[1:-1].replace(",", ""): (t, kind)
            for k in ("int3c", "deriv3c") for t, c, _n, kind in res[k]["top"]}


def measure(workloads: list[str]) -> dict:
    base = {w: _times(w, None) for w in workloads}
    var = {w: _times(w, VARIANT) for w in workloads}
    choice, detail = {}, {}
    keys = sorted({k for w in workloads for k, (_t, kind) in base[w].items() if kind != "warp"})
    for k in keys:
        gains = [1.0 - var[w][k][0] / base[w][k][0] for w in workloads if k in base[w] and k in var[w]]
        detail[k] = [round(g, 3) for g in gains]
        if gains and min(gains) >= MIN_GAIN:
            choice[k] = 4
    import torch

    return {"min_blocks": choice, "gain_by_class": detail, "workloads": workloads,
            "device": torch.cuda.get_device_name(0), "min_gain": MIN_GAIN}


def main() -> None:
    if len(sys.argv) < 2 or sys.argv[1] not in ("build", "measure"):
        raise SystemExit(__doc__)
    if sys.argv[1] == "build":
        from .build import build_variant

        print(build_variant(["DFB_THREAD_MIN_BLOCKS=4"], VARIANT, "minb4"))
        return
    args = sys.argv[2:]
    out = None
    if "--out" in args:
        i = args.index("--out")
        out = args[i + 1]
        args = args[:i] + args[i + 2:]
    res = measure(args or ["w8"])
    text = json.dumps(res, indent=1, sort_keys=True)
    if out:
        with open(out, "w") as f:
            f.write(text + "\n")
    print(text)


if __name__ == "__main__":
    main()
