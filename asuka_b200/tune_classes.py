"""Measured per-class kernel shapes for the class-specialised Rys kernels (the autotuner).

Two knobs are tuned per angular class, each against the default build:

* launch bounds: the thread kernels run 128 threads per block and may take up to 255
  registers (the classes use 150-170, i.e. 3 resident blocks per SM); capping them at 128
  (4 blocks per SM) helps the classes whose working set still fits and hurts those that spill
  (variant "minb4");
* the aux-component split: a class is split over FS threads per task so that one thread's
  accumulators fit a register budget; every extra split repeats the task's Rys roots and
  recurrence tables, a larger budget (fewer, heavier threads) trades that against registers
  (variants "acc100" and "acc136": derivative budgets 100 and 136 doubles instead of 66,
  integral budgets 64 and 96 instead of 40); a larger budget also moves classes from the
  generic warp path onto the thread kernels.

Which is better is measured, not guessed:

    python -m asuka_b200.tune_classes build                   # (no GPU) the variant libraries
    python -m asuka_b200.tune_classes measure w8 w4q --out T  # (GPU) time every class with each library
    cp T asuka_b200/csrc/class_tuning.json && python asuka_b200/csrc/gen_classes.py && python -m asuka_b200.build

A class takes a variant when it is at least ``MIN_GAIN`` faster with it on every workload
that contains the class (the fastest qualifying variant wins); ``gen_classes.py`` reads the
table when generating the kernels.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
VARIANTS = {
    "minb4": dict(defines=["DFB_THREAD_MIN_BLOCKS=4"], gen_env=None,
                  table=("min_blocks", 4)),
    "acc100": dict(defines=[], gen_env={"DFB_GEN_NO_TUNING": "1", "DFB_GEN_ACC_BUDGET_DERIV": "100",
                                        "DFB_GEN_ACC_BUDGET_INT": "64"},
                   table=("acc_budget", None)),
    "acc136": dict(defines=[], gen_env={"DFB_GEN_NO_TUNING": "1", "DFB_GEN_ACC_BUDGET_DERIV": "136",
                                        "DFB_GEN_ACC_BUDGET_INT": "96"},
                   table=("acc_budget", None)),
}
# accumulator budgets of the generated variants (derivative, integral classes)
_BUDGETS = {"acc100": (100, 64), "acc136": (136, 96)}
MIN_GAIN = 0.03


def _lib(name: str) -> str:
    return os.path.join(HERE, "_tune", f"libdfb_{name}.so")


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
    """Time every class with the untuned default build and with each variant; the default build
    must be generated without a tuning table (``DFB_GEN_NO_TUNING=1``) for a clean baseline."""
    base = {w: _times(w, None) for w in workloads}
    var = {v: {w: _times(w, _lib(v)) for w in workloads} for v in VARIANTS}
    table = {"min_blocks": {}, "acc_budget": {}}
    detail = {}
    keys = sorted({k for w in workloads for k in base[w]})
    for k in keys:
        best = None
        for v, times in var.items():
            gains = [1.0 - times[w][k][0] / base[w][k][0] for w in workloads if k in base[w] and k in times[w]]
            detail.setdefault(k, {})[v] = [round(g, 3) for g in gains]
            if gains and min(gains) >= MIN_GAIN and (best is None or min(gains) > best[1]):
                best = (v, min(gains))
        if best is not None:
            field, value = VARIANTS[best[0]]["table"]
            if value is None:  # generated variant: the class's budget in that variant
                value = _BUDGETS[best[0]][0 if k.startswith("d") else 1]
            table[field][k] = value
    import torch

    return {**table, "gain_by_class": detail, "workloads": workloads,
            "device": torch.cuda.get_device_name(0), "min_gain": MIN_GAIN}


def main() -> None:
    if len(sys.argv) < 2 or sys.argv[1] not in ("build", "measure"):
        raise SystemExit(__doc__)
    if sys.argv[1] == "build":
        from .build import build_variant

        for v, spec in VARIANTS.items():
            print(build_variant(spec["defines"], _lib(v), v, gen_env=spec["gen_env"]))
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
