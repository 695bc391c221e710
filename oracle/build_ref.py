"""Compile the reference's own CUDA extension (FL/cuda_lib) from its sources,
unmodified, into ``oracle/_ref/`` so the GPU tests can use it as a second
checker and as a golden-vector generator.

Test infrastructure only: nothing in the product imports this.  The sources
are read from the reference checkout (``ref_root()``: the ``FL_REF_ROOT``
environment variable, else the read-only checkout this recipe was written
against) and only the built ``.so`` lands in ``oracle/_ref``; the
reference's own ``setup.py`` is not used.  Build flags: ``-O2`` as in the
reference's ``setup.py:19-21`` plus an explicit sm_100a target.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
NAME = "ref_atten_cuda"
# where the reference checkout is mounted read-only on the build machine; the
# GPU machines have no checkout and use the prebuilt .so
DEFAULT_REF_ROOT = "/root/reference"


def ref_root(required=False):
    """The reference checkout: FL_REF_ROOT if set, else DEFAULT_REF_ROOT.
    Returns None (or raises, with required=True) when neither holds FL/."""
    root = os.environ.get("FL_REF_ROOT") or DEFAULT_REF_ROOT
    if os.path.isdir(os.path.join(root, "FL")):
        return root
    if required:
        raise FileNotFoundError(
            "reference checkout not found at %r: set FL_REF_ROOT to the FL_correction "
            "checkout (the directory that holds FL/)" % root)
    return None


def build(verbose=False):
    src_dir = os.path.join(ref_root(required=True), "FL", "cuda_lib")
    srcs = [os.path.join(src_dir, "atten_cuda.cpp"), os.path.join(src_dir, "atten_cuda_kernel.cu")]
    if not all(os.path.exists(s) for s in srcs):
        raise FileNotFoundError("reference sources not found under %s" % src_dir)
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    from torch.utils.cpp_extension import load
    load(name=NAME, sources=srcs, build_directory=OUT,
         extra_cflags=["-O2"],
         extra_cuda_cflags=["-O2", "-gencode=arch=compute_100a,code=sm_100a"],
         verbose=verbose, is_python_module=True)
    return os.path.join(OUT, NAME + ".so")


def load_built():
    """Import the prebuilt reference extension from ``oracle/_ref``."""
    import importlib.util
    import torch  # noqa: F401  (the extension links against libtorch)
    path = os.path.join(OUT, NAME + ".so")
    spec = importlib.util.spec_from_file_location(NAME, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
