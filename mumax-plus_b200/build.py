"""Build libmpx.so (the sm_100a engine behind include/mpx.h) in-tree with nvcc.

The library is one translation unit (csrc/engine.cu includes the kernel
headers) compiled for sm_100a only.  The resulting shared object sits next to
this file so that it travels with the source tree.  A second build of the same
sources with -DMPX_BOUNDS_CHECK, libmpx_checked.so, verifies the index of every
per-cell field access (mpx_bounds_check reads the record); the two compile in
parallel.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "engine.cu")
HEADERS = sorted(os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc")) if f.endswith(".cuh"))
OUT = os.path.join(HERE, "libmpx.so")
OUT_CHECKED = os.path.join(HERE, "libmpx_checked.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date(out=OUT):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    deps = [SRC, os.path.join(ROOT, "include", "mpx.h"), __file__] + HEADERS
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _command(out, extra):
    defs = ["-DMPX_BOUNDS_CHECK"] if out == OUT_CHECKED else []
    return [nvcc_path()] + NVCC_FLAGS + defs + list(extra) + ["-I", os.path.join(ROOT, "include"), SRC, "-o", out]


def build(force=False, verbose=False, extra=(), checked=True):
    """Compile libmpx.so (and libmpx_checked.so when `checked`) for sm_100a;
    returns the path of libmpx.so."""
    outs = [o for o in ([OUT, OUT_CHECKED] if checked else [OUT]) if force or not up_to_date(o)]
    procs = []
    for out in outs:
        cmd = _command(out, extra)
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    errors = []
    for proc in procs:
        so, se = proc.communicate()
        if proc.returncode != 0:
            errors.append(so + se)
        elif verbose and (so or se):
            print(so + se, file=sys.stderr)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    return OUT


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=force or bool(extra), verbose=True, extra=extra))
