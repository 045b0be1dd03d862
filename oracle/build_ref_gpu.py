"""Build recipe for the reference's own GPU scan kernels (test and baseline
infrastructure; the package never loads what this builds).

Reads the CUDA source strings ``_SRC_SCALED`` from the reference checkout
(whyihaveyou/rgs70-classical-challenge: work/rgs_attack/upstream_scan/gpu_kernel.py for
complex64 and gpu_kernel_fp64.py for complex128) where they lie, writes each with this
directory's host loop (ref_gpu_launcher.cuh) into ``oracle/_ref/`` and compiles them
with nvcc for sm_100a into ``oracle/_ref/libref_scan_c64.so`` / ``libref_scan_c128.so``.
Nothing of the reference is copied into the repository: ``oracle/_ref/`` is git-ignored.

    python oracle/build_ref_gpu.py [--reference PATH]

The reference is looked up in --reference, then $RGS_REFERENCE, then /root/reference;
without it the recipe does nothing (the GPU box uses the files built here).
"""
import ast
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
SOURCES = {"c64": "gpu_kernel.py", "c128": "gpu_kernel_fp64.py"}


def reference_root(argv=()):
    argv = list(argv)
    if "--reference" in argv and argv.index("--reference") + 1 < len(argv):
        return Path(argv[argv.index("--reference") + 1])
    return Path(os.environ.get("RGS_REFERENCE", "/root/reference"))


def kernel_source(path):
    """The value of the module-level string ``_SRC_SCALED`` (parsed, not executed)."""
    tree = ast.parse(Path(path).read_text())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "_SRC_SCALED" for t in node.targets):
            return ast.literal_eval(node.value)
    raise ValueError(f"_SRC_SCALED not found in {path}")


def build(reference=None, verbose=False):
    """Compile both libraries; returns their paths, or {} when the reference is absent."""
    ref = Path(reference) if reference else reference_root()
    src_dir = ref / "work" / "rgs_attack" / "upstream_scan"
    if not src_dir.is_dir():
        return {}
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    OUT.mkdir(exist_ok=True)
    out = {}
    for prec, name in SOURCES.items():
        cu = OUT / f"ref_scan_{prec}.cu"
        lib = OUT / f"libref_scan_{prec}.so"
        text = kernel_source(src_dir / name)
        body = ("// Generated by oracle/build_ref_gpu.py from the reference's " + name + " (not in the repository).\n"
                + ("#define REF_C128 1\n" if prec == "c128" else "") + text
                + f'\n#include "{HERE / "ref_gpu_launcher.cuh"}"\n')
        if not cu.exists() or cu.read_text() != body or not lib.exists() or \
                lib.stat().st_mtime < (HERE / "ref_gpu_launcher.cuh").stat().st_mtime:
            cu.write_text(body)
            cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared", "-Xcompiler", "-fPIC",
                   "-o", str(lib), str(cu)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        out[prec] = lib
    return out


if __name__ == "__main__":
    print(build(reference_root(sys.argv[1:]), verbose=True))
