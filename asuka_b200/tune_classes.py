"""Measured per-class kernel shapes for the class-specialised Rys kernels (the autotuner).

Three knobs are tuned per angular class, each against the default build:

* launch bounds: the thread kernels run 128 threads per block and may take up to 255
  registers (many classes use 180-230, i.e. 2 resident blocks per SM); capping them at 170
  (3 blocks per SM, variant "minb3") or 128 (4 blocks, "minb4") helps the classes whose
  working set still fits and hurts those that spill;
* the aux-component split: a class is split over FS threads per task so that one thread's
  live accumulators fit a register budget; every extra split repeats the task's Rys roots
  and recurrence tables, a larger budget (fewer, heavier threads) trades that against
  registers and parallelism (variants "acc64"/"acc96": integral budgets 64 and 96 doubles
  instead of 40; "dacc56"/"dacc72"/"dacc96"/"dacc128": derivative budgets instead of 40); a larger
  budget also moves classes from the generic warp path onto the thread kernels;
* Rys-table staging ("stage1"): classes of at most 3 roots copy their root count's coefficient
  table into shared memory once per block (one bulk asynchronous copy) and gather from there;
  this costs shared memory, and so occupancy, in the classes that fit several blocks per SM.

Which is better is measured, not guessed.  A tuning pass covers one kind of knob (``--set``)
and keeps the table's other entries:

    python -m asuka_b200.tune_classes build --set deriv          # (no GPU) the variant libraries
    python -m asuka_b200.tune_classes measure w8 w4q --set deriv --out T   # (GPU) time every class
    cp T asuka_b200/csrc/class_tuning.json && python asuka_b200/csrc/gen_classes.py && python -m asuka_b200.build

or, one library per GPU run (``times``), then the selection on any machine (``select``):

    python -m asuka_b200.tune_classes times w8 w4q --out base.json              # (GPU) default build
    python -m asuka_b200.tune_classes times w8 w4q --lib dacc56 --out v56.json  # (GPU) one variant
    python -m asuka_b200.tune_classes select --set deriv --base base.json --var dacc56=v56.json ... --out T

The default build the variants are measured against must be generated without the table's
entries of the set being tuned (``strip``: ``python -m asuka_b200.tune_classes strip --set
deriv``, then regenerate and build).  A class takes a variant when it is at least ``MIN_GAIN``
faster with it on every workload that contains the class (the fastest qualifying variant
wins); ``gen_classes.py`` reads the table when generating the kernels.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# set -> variants; a variant is (extra -D flags, generator environment, table entry it selects).
# The "int" and "deriv" variants override the budget of every class of that kind and keep the
# table's entries for the other kind.
VARIANTS = {
    "launch": {
        "minb3": dict(defines=["DFB_THREAD_MIN_BLOCKS=3"], gen_env=None, table=("min_blocks", 3)),
        "minb4": dict(defines=["DFB_THREAD_MIN_BLOCKS=4"], gen_env=None, table=("min_blocks", 4)),
    },
    "int": {
        "acc64": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_INT": "64"}, table=("acc_budget", 64)),
        "acc96": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_INT": "96"}, table=("acc_budget", 96)),
    },
    "deriv": {
        "dacc56": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_DERIV": "56"}, table=("acc_budget", 56)),
        "dacc72": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_DERIV": "72"}, table=("acc_budget", 72)),
        "dacc96": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_DERIV": "96"}, table=("acc_budget", 96)),
        "dacc128": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_DERIV": "128"}, table=("acc_budget", 128)),
    },
    # the Rys table copied into shared memory per block (classes of at most 3 roots); one variant
    # library serves both sets: "stage" times the FP64 kernels, "f32stage" the FP32 ones
    "stage": {
        "stage1": dict(defines=[], gen_env={"DFB_GEN_STAGE": "1"}, table=("stage", 1)),
    },
    "f32stage": {
        "stage1": dict(defines=[], gen_env={"DFB_GEN_STAGE": "1"}, table=("stage_f32", 1)),
    },
    # the mixed-precision derivative kernels (float accumulators: budgets count floats), timed in FP32;
    # larger uniform budgets make the (f d|.) files compile for over 40 minutes each
    "f32deriv": {
        "fd112": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_DERIV_F32": "112"}, table=("acc_budget_f32", 112)),
        "fd144": dict(defines=[], gen_env={"DFB_GEN_ACC_BUDGET_DERIV_F32": "144"}, table=("acc_budget_f32", 144)),
    },
}
# precision the classes of a set are timed in
_PRECISION = {"f32deriv": "mixed_all", "f32stage": "mixed_all"}
# the table entries a set owns: (field, class-key prefix)
_OWNS = {"launch": ("min_blocks", ""), "int": ("acc_budget", "i"), "deriv": ("acc_budget", "d"),
         "f32deriv": ("acc_budget_f32", "d"), "stage": ("stage", ""), "f32stage": ("stage_f32", "")}
MIN_GAIN = 0.03
TABLE = os.path.join(HERE, "csrc", "class_tuning.json")


def _lib(name: str) -> str:
    return os.path.join(HERE, "_tune", f"libdfb_{name}.so")


def _times(workload: str, lib: str | None, precision: str = "fp64") -> dict:
    env = dict(os.environ)
    env.pop("DFB_LIB_PATH", None)
    if lib:
        env["DFB_LIB_PATH"] = lib
    code = ("import json; from asuka_b200.profile_step import setup, class_times; "
            f"mol, eng, Cw, R = setup({workload!r}); "
            f"print(json.dumps(class_times(eng, mol, top=10000, precision={precision!r})))")
    out = subprocess.run([sys.executable, "-c", code], env=env, check=True, capture_output=True, text=True,
                         cwd=os.path.dirname(HERE)).stdout
    res = json.loads(out.strip().splitlines()[-1])
    return {("d" if k == "deriv3c" else "i") + c[1:-1].replace(",", ""): (t, kind)
            for k in ("int3c", "deriv3c") for t, c, _n, kind in res[k]["top"]}


def _load_table() -> dict:
    if not os.path.exists(TABLE):
        return {"min_blocks": {}, "acc_budget": {}}
    with open(TABLE) as f:
        return json.load(f)


def strip(tset: str) -> dict:
    """The current table without the entries owned by ``tset`` (the default build to measure against)."""
    table = _load_table()
    field, prefix = _OWNS[tset]
    table[field] = {k: v for k, v in table.get(field, {}).items() if not k.startswith(prefix)}
    table.setdefault("acc_budget", {})
    table.setdefault("min_blocks", {})
    return table


def measure(workloads: list[str], tset: str) -> dict:
    """Time every class with the default build (generated from ``strip(tset)``) and with each
    variant of the set; the table's entries outside the set are kept."""
    prec = _PRECISION.get(tset, "fp64")
    base = {w: _times(w, None, prec) for w in workloads}
    var = {v: {w: _times(w, _lib(v), prec) for w in workloads} for v in VARIANTS[tset]}
    return select(base, var, tset)


def select(base: dict, var: dict, tset: str) -> dict:
    """The table from measured class times: ``base[workload][class] = (ms, kind)`` of the default
    build and ``var[variant][workload][class]`` of each variant."""
    workloads = sorted(base)
    variants = VARIANTS[tset]
    table = strip(tset)
    field, prefix = _OWNS[tset]
    table.setdefault(field, {})
    detail = {}
    keys = sorted({k for w in workloads for k in base[w] if k.startswith(prefix)})
    for k in keys:
        best = None
        for v, times in var.items():
            gains = [1.0 - times[w][k][0] / base[w][k][0] for w in workloads if k in base[w] and k in times[w]]
            detail.setdefault(k, {})[v] = [round(g, 3) for g in gains]
            if gains and min(gains) >= MIN_GAIN and (best is None or min(gains) > best[1]):
                best = (v, min(gains))
        if best is not None:
            f, value = variants[best[0]]["table"]
            table[f][k] = value
    gains = dict(table.get("gain_by_class", {}))
    for k, d in detail.items():  # variant names are unique over the sets: merge per class
        gains[k] = {**gains.get(k, {}), **d}
    table.update(gain_by_class=gains, min_gain=MIN_GAIN)
    table.setdefault("workloads", workloads)
    table.setdefault("tuned_sets", {})[tset] = workloads
    return table


def main() -> None:
    if len(sys.argv) < 2 or sys.argv[1] not in ("build", "measure", "strip", "times", "select"):
        raise SystemExit(__doc__)
    args = sys.argv[2:]
    tset = "deriv"
    if "--set" in args:
        i = args.index("--set")
        tset = args[i + 1]
        args = args[:i] + args[i + 2:]
    if tset not in VARIANTS:
        raise SystemExit(f"--set must be one of {sorted(VARIANTS)}")
    if sys.argv[1] == "times":  # one library per run: the variant libraries are large
        lib = None
        if "--lib" in args:
            i = args.index("--lib")
            lib = args[i + 1] if args[i + 1].endswith(".so") else _lib(args[i + 1])
            args = args[:i] + args[i + 2:]
        i = args.index("--out")
        out, args = args[i + 1], args[:i] + args[i + 2:]
        import torch

        prec = _PRECISION.get(tset, "fp64")
        res = {"device": torch.cuda.get_device_name(0), "precision": prec,
               "times": {w: {k: list(v) for k, v in _times(w, lib, prec).items()} for w in args or ["w8"]}}
        with open(out, "w") as f:
            json.dump(res, f)
        return
    if sys.argv[1] == "select":  # --base B.json --var NAME=F.json ... --out T
        def grab(flag):
            vals = []
            while flag in args:
                i = args.index(flag)
                vals.append(args[i + 1])
                del args[i:i + 2]
            return vals

        def load(path):
            with open(path) as f:
                d = json.load(f)
            return {w: {k: tuple(v) for k, v in t.items()} for w, t in d["times"].items()}, d["device"]

        base, device = load(grab("--base")[0])
        var = {}
        for spec in grab("--var"):
            name, path = spec.split("=", 1)
            var[name] = load(path)[0]
        out = grab("--out")[0]
        res = select(base, var, tset)
        res["device"] = device
        with open(out, "w") as f:
            f.write(json.dumps(res, indent=1, sort_keys=True) + "\n")
        return
    if sys.argv[1] == "build":
        from .build import build_variant

        for v, spec in VARIANTS[tset].items():
            print(build_variant(spec["defines"], _lib(v), v, gen_env=spec["gen_env"]))
        return
    if sys.argv[1] == "strip":
        text = json.dumps(strip(tset), indent=1, sort_keys=True) + "\n"
        with open(TABLE, "w") as f:
            f.write(text)
        return
    out = None
    if "--out" in args:
        i = args.index("--out")
        out = args[i + 1]
        args = args[:i] + args[i + 2:]
    res = measure(args or ["w8"], tset)
    import torch

    res["device"] = torch.cuda.get_device_name(0)
    text = json.dumps(res, indent=1, sort_keys=True)
    if out:
        with open(out, "w") as f:
            f.write(text + "\n")
    print(text)


if __name__ == "__main__":
    main()
