"""Build the CUDA library in-tree: ``prince_b200/libprince_b200.so`` for sm_100a.

``python -m prince_b200.build`` (or ``build()``) runs nvcc on
``prince_b200/csrc/prince_b200.cu``.  The library is rebuilt when any source
is newer than the ``.so``.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(HERE, "libprince_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "prince_b200.cu")]
GENCODE = "arch=compute_100a,code=sm_100a"


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build():
    if not os.path.exists(SO):
        return True
    deps = SOURCES + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "prince_b200.h")]
    t = os.path.getmtime(SO)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return SO
    cmd = [_nvcc(), "-gencode", GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-shared", "-o", SO + ".tmp", *SOURCES]
    if verbose:
        cmd.append("-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(SO + ".tmp", SO)
    return SO


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
