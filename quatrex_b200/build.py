"""Build libqtxrgf.so in-tree for sm_100a with nvcc (no JIT cache, no torch types).

``python -m quatrex_b200.build`` compiles every ``csrc/*.cu`` into
``quatrex_b200/libqtxrgf.so``.  The library travels with the source tree.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libqtxrgf.so")
# the FP64 peak probe of kernel_bench (a measurement tool, kept out of libqtxrgf.so)
PROBE_SRC = os.path.join(HERE, "probe", "peak_probe.cu")
PROBE_LIB = os.path.join(HERE, "libqtxprobe.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _stale(lib: str, deps: list[str]) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(d) > t for d in deps)


def build_probe(force: bool = False) -> str:
    if force or _stale(PROBE_LIB, [PROBE_SRC]):
        tmp = PROBE_LIB + ".tmp"
        subprocess.check_call([nvcc_path(), *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                               "-cudart", "static", PROBE_SRC, "-o", tmp])
        os.replace(tmp, PROBE_LIB)
    return PROBE_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h"))
    deps += glob.glob(os.path.join(ROOT, "include", "*.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c", src, "-o", obj,
               "-I", os.path.join(ROOT, "include")]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_probe(force="--force" in sys.argv))
