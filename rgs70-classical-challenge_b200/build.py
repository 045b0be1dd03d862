"""Build the native library ``librgs_b200.so`` in-tree with nvcc for sm_100a.

Every ``csrc/*.cu`` and ``csrc/*.cpp`` is compiled to an object under ``_build/``
(at the repository root, git-ignored) and linked into
``<package>/librgs_b200.so``.  Objects are rebuilt when their source or any
header is newer.  Needs nvcc but no GPU (cross-compilation).
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "librgs_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-I", str(CSRC), "-I", str(INCLUDE)]
# Extra nvcc flags (launch-shape knobs such as -DRGS_PAIR_MINB=3 for tuning builds).
FLAGS += os.environ.get("RGS_NVCC_FLAGS", "").split()


def _nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA library cannot be built")
    return exe


def _newest_header():
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(verbose=False, ptxas_info=False, jobs=None):
    """Compile and link; returns the library path."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    hdr = _newest_header()
    objs, cmds = [], []
    for src in sources:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr) and not ptxas_info:
            continue
        cmd = [nvcc, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        if ptxas_info and src.suffix == ".cu":
            cmd += ["-Xptxas", "-v"]
        cmds.append(cmd)
    procs = []
    jobs = jobs or min(8, os.cpu_count() or 1)
    for cmd in cmds:
        while len(procs) >= jobs:
            _reap(procs, verbose or ptxas_info)
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    while procs:
        _reap(procs, verbose or ptxas_info)
    if cmds or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        link = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs), "-lcuda"]
        if verbose:
            print(" ".join(link), flush=True)
        subprocess.run(link, check=True)
    return LIB


def _reap(procs, show):
    cmd, p = procs.pop(0)
    out, _ = p.communicate()
    if p.returncode != 0:
        sys.stderr.write(out)
        raise RuntimeError("nvcc failed: " + " ".join(cmd[-3:]))
    if show and out.strip():
        sys.stdout.write(out)


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
