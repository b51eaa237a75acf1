"""Build the in-tree shared library ``libafr_b200.so`` for sm_100a with nvcc.

``python -m autoflowcfd_b200.build`` (or ``__graft_entry__.build()``) compiles
every CUDA source under ``csrc/`` into one C-ABI library next to this file.
nvcc cross-compiles without a GPU.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libafr_b200.so")
SOURCES = ["afr_api.cu", "afr_tc_check.cu", "afr_facegeom.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-source flags: the flux-point construction rounds every product and sum
# separately, as the reference's numpy / Numba code does (no multiply-add
# contraction)
SOURCE_FLAGS = {"afr_facegeom.cu": ["-fmad=false"]}


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources_newer_than_lib():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for root, _, files in os.walk(CSRC):
        for f in files:
            if os.path.getmtime(os.path.join(root, f)) > t:
                return True
    inc = os.path.join(os.path.dirname(HERE), "include", "afr_b200.h")
    return os.path.exists(inc) and os.path.getmtime(inc) > t


def build(force=False, verbose=False, extra=None):
    """Compile libafr_b200.so; returns its path."""
    if not force and not sources_newer_than_lib():
        return LIB
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    common = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *(extra or [])]
    with tempfile.TemporaryDirectory(prefix="afr_build_") as tmp:
        objs = [os.path.join(tmp, os.path.splitext(src)[0] + ".o") for src in SOURCES]
        cmds = [common + SOURCE_FLAGS.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
                for src, obj in zip(SOURCES, objs)]
        cmds.append([nvcc_path(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"])

        def run(cmd):
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
            if verbose and (r.stdout or r.stderr):
                print(r.stdout + r.stderr)

        with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
            list(pool.map(run, cmds[:-1]))
        run(cmds[-1])
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, extra=["-Xptxas", "-v"] if "-v" in sys.argv else None))
