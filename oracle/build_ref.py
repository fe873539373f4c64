"""Compile the reference's CPU Rys kernels (ORACLE / CPU-baseline use only).

Cythonises ``asuka/cueri/_eri_rys_cpu.pyx`` where it lies in the reference
checkout (never copied into this repository) with the reference's own build
settings -- ``CY_K_LMAX`` compile-time constant (8 here, for l <= 8 aux
shells), ``-O3 -fopenmp -DCUERI_USE_OPENMP=1`` (reference ``setup.py:103-132,
180-192``) -- and writes the generated C and the extension module only into
``oracle/_ref/``.  The module is imported as ``_eri_rys_cpu`` by the checker
and by the CPU-baseline arm of ``bench.py``; it is never part of the product.

    python oracle/build_ref.py [reference_root]
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def main(ref_root: str = "/root/reference") -> int:
    pyx = os.path.join(ref_root, "asuka", "cueri", "_eri_rys_cpu.pyx")
    if not os.path.exists(pyx):
        print(f"reference source not found: {pyx}", file=sys.stderr)
        return 1
    import numpy as np

    os.makedirs(OUT, exist_ok=True)
    c_file = os.path.join(OUT, "_eri_rys_cpu.c")
    so = os.path.join(OUT, "_eri_rys_cpu" + sysconfig.get_config_var("EXT_SUFFIX"))
    subprocess.run([sys.executable, "-m", "cython", "-3", "-E", "CY_K_LMAX=8", "--module-name", "_eri_rys_cpu",
                    pyx, "-o", c_file], check=True)
    subprocess.run(["gcc", "-O3", "-fopenmp", "-shared", "-fPIC", "-DCUERI_USE_OPENMP=1",
                    "-DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION", f"-I{sysconfig.get_paths()['include']}",
                    f"-I{np.get_include()}", c_file, "-o", so, "-lm"], check=True)
    print(so)
    return 0


if __name__ == "__main__":
    sys.exit(main(*sys.argv[1:]))
