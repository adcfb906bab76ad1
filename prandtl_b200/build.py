"""Build the sm_100a shared library libprandtl_b200.so in-tree with nvcc.

Usage: python -m prandtl_b200.build [--verbose-ptxas]
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libprandtl_b200.so")
SOURCES = (["dgsem_kernels.cu", "prandtl_api.cu", "prandtl_noalloc.cu", "prandtl_batch.cu", "prandtl_serve.cu",
            "prandtl_mesh.cu", "prandtl_io.cu"] +
           sorted(os.path.basename(p) for p in glob.glob(os.path.join(CSRC, "dgsem_inst_*.cu"))))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "prandtl_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose_ptxas: bool = False, force: bool = False, lib: str = LIB, defines=()) -> str:
    """Compile the sources into `lib` (default: the in-tree library).  `defines`
    are extra -D flags (launch-shape overrides used when tuning)."""
    if not force and lib == LIB and not needs_build():
        return LIB
    tag = "" if lib == LIB else f".{abs(hash(lib)) % 100000}"

    def compile_one(src):
        obj = os.path.join(CSRC, src.replace(".cu", f"{tag}.o"))
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", *[f"-D{d}" for d in defines],
               "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    # heaviest translation units first so the parallel build ends together
    order = sorted(SOURCES, key=lambda f: (not f.startswith("dgsem_inst_d3"), f))
    objs, failed = [], []
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for src, obj, r in ex.map(compile_one, order):
            if r.stdout or r.stderr:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(src)
            objs.append(obj)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return lib


if __name__ == "__main__":
    build(verbose_ptxas="--verbose-ptxas" in sys.argv, force=True)
    print(LIB)
