"""Build recipe for the native library ``fl_correction_b200/libflc.so``.

    python -m fl_correction_b200.build

Compiles every ``csrc/*.cu`` for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) with nvcc and links one shared library that
exports the C ABI of ``include/flc.h``.  The library depends on the CUDA
runtime only (no torch), so any FFI can bind it.
"""
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libflc.so")
BUILD = os.path.join(PKG, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h")))


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in sources() + headers() + [__file__])


def build(force=False, verbose=False, extra_flags=()):
    """Compile and link libflc.so if any source is newer than it."""
    if not force and not stale():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc(), "-c", src, "-o", obj, "-I", os.path.join(ROOT, "include")] + NVCC_FLAGS + list(extra_flags)
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            print(text)
    if failed:
        msg = "\n".join("%s:\n%s" % f for f in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    tmp = OUT + ".tmp"
    link = [nvcc(), "-shared", "-o", tmp] + objs + ["-gencode", "arch=compute_100a,code=sm_100a", "-lcudart"]
    subprocess.check_call(link)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv,
                extra_flags=[a for a in sys.argv[1:] if a.startswith("-X") or a.startswith("--ptxas")]))
