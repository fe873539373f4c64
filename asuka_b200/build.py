"""Build ``libdfb.so`` in place with nvcc for sm_100a.

    python -m asuka_b200.build
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdfb.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "--shared",
              "-Xcompiler", "-fPIC", "-lcublas"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    """True when the library is missing or older than a source, a header a source includes, or
    when a source has no object yet."""
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    objdir = os.path.join(HERE, "_build")
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        if not os.path.exists(obj) or os.path.getmtime(obj) > t:
            return True
        if any(os.path.getmtime(p) > t for p in [src, *_local_includes(src)]):
            return True
    return False


def _local_includes(path: str, seen: set | None = None) -> set:
    """Headers of this source tree that ``path`` includes, directly or through other headers
    (#include "..." lines), so that a header change rebuilds only the objects that use it."""
    import re

    seen = set() if seen is None else seen
    try:
        with open(path) as f:
            txt = f.read()
    except OSError:
        return seen
    for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', txt, flags=re.M):
        h = os.path.normpath(os.path.join(os.path.dirname(path), name))
        if h not in seen and os.path.exists(h):
            seen.add(h)
            _local_includes(h, seen)
    return seen


def _same_as_main(src: str, srcdir: str) -> bool:
    """True when ``src`` (in a generated copy of csrc) and every header it includes from that
    copy are byte-identical to the main tree's files, whose object is then up to date."""

    def read(p):
        with open(p, "rb") as f:
            return f.read()

    for p in [src, *_local_includes(src)]:
        rel = os.path.relpath(p, srcdir)
        main = os.path.normpath(os.path.join(CSRC, rel))
        if not os.path.exists(main) or read(p) != read(main):
            return False
    return os.path.exists(os.path.join(HERE, "_build", os.path.basename(src)[:-3] + ".o"))


def _wait_slot(procs: list, jobs: int) -> None:
    """Block until fewer than ``jobs`` of the compiler processes are still running."""
    while sum(1 for p in procs if p.poll() is None) >= jobs:
        time.sleep(0.2)


def _flags_changed(objdir: str, flags: list[str]) -> bool:
    p = os.path.join(objdir, "flags.txt")
    if not os.path.exists(p):
        return True
    with open(p) as f:
        return f.read() != " ".join(flags)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    """Compile every csrc/*.cu to an object in parallel (they are independent), then link."""
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f not in ("--shared", "-lcublas")]
    procs = []
    objs = []
    jobs = jobs or max(1, os.cpu_count() or 1)
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        t_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _local_includes(src)])
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= t_dep
                and not _flags_changed(objdir, compile_flags)):
            continue
        cmd = [nvcc, *compile_flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        _wait_slot(procs, jobs)
        procs.append(subprocess.Popen(cmd, cwd=CSRC))
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed: {p.args}")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-o", OUT + ".tmp", *objs],
                   check=True, cwd=CSRC)
    with open(os.path.join(objdir, "flags.txt"), "w") as f:
        f.write(" ".join(compile_flags))
    os.replace(OUT + ".tmp", OUT)
    return OUT


def build_variant(defines: list[str], out: str, tag: str, jobs: int | None = None,
                  gen_env: dict | None = None) -> str:
    """A second library for the class tuner (objects in _build_<tag>).

    ``defines``: extra -D flags for the class-specialised kernels, the other sources reuse
    the main build's objects.  ``gen_env``: regenerate the class kernels under these
    environment variables (e.g. another accumulator budget) in a copy of csrc and build the
    sources of that copy; a source whose text and included headers are byte-identical to the
    main tree's reuses the main build's object.
    """
    import shutil

    build()
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(HERE, "_build")
    vdir = os.path.join(HERE, f"_build_{tag}")
    os.makedirs(vdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f not in ("--shared", "-lcublas")] + [f"-D{d}" for d in defines]
    # the sources include "../../include/dfb.h" relative to csrc: -I csrc resolves it for the copy too
    inc = ["-I", CSRC]
    srcdir = CSRC
    if gen_env:
        srcdir = os.path.join(vdir, "src")
        if os.path.exists(srcdir):
            shutil.rmtree(srcdir)
        shutil.copytree(CSRC, srcdir, ignore=shutil.ignore_patterns("__pycache__"))
        env = dict(os.environ, **gen_env)
        subprocess.run([sys.executable, os.path.join(srcdir, "gen_classes.py"), srcdir], check=True, env=env)
    objs, procs = [], []
    jobs = jobs or max(1, os.cpu_count() or 1)
    for src in sorted(glob.glob(os.path.join(srcdir, "*.cu"))):
        base = os.path.basename(src)[:-3]
        if (not gen_env and not base.startswith("dfb_cls_")) or (gen_env and not defines
                                                                 and _same_as_main(src, srcdir)):
            objs.append(os.path.join(objdir, base + ".o"))
            continue
        obj = os.path.join(vdir, base + ".o")
        objs.append(obj)
        _wait_slot(procs, jobs)
        procs.append(subprocess.Popen([nvcc, *compile_flags, *inc, "-c", src, "-o", obj], cwd=srcdir))
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed: {p.args}")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-o", out, *objs],
                   check=True, cwd=srcdir)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
