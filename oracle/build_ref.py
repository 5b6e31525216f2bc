"""Compile the reference's own CUDA projector (test infrastructure only).

    python oracle/build_ref.py            # needs the reference checkout

Builds src/bindings.cpp, src/ct_projector_2d.cu and src/ct_projector_3d.cu
from the read-only reference checkout ($CTLAB_REFERENCE, else the checkout
beside this repository: oracle/reference_path.py) into oracle/_ref/ctlab_ref_C*.so as a torch extension named
``ctlab_ref_C`` (the reference's ``ct_laboratory._C`` under another name),
with the flags of its setup.py (-O2) and the sm_100 target of its benchmark
image (benchmark/Dockerfile:11, TORCH_CUDA_ARCH_LIST=10.0).  No reference
source is copied into this repository; the built library is git-ignored and
travels to the GPU box with the working tree.  GPU tests load it with
``load_ref()`` to compare against the reference's kernels on identical
inputs.
"""
from __future__ import annotations

import glob
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def built_path():
    hits = sorted(glob.glob(os.path.join(OUT, "ctlab_ref_C*.so")))
    return hits[0] if hits else None


def build(verbose=True):
    from torch.utils.cpp_extension import load
    try:
        from oracle.reference_path import reference_root
    except ImportError:  # run as a script from oracle/
        from reference_path import reference_root
    REF = reference_root(required=True)
    src = [os.path.join(REF, "src", f) for f in ("bindings.cpp", "ct_projector_2d.cu", "ct_projector_3d.cu")]
    missing = [s for s in src if not os.path.exists(s)]
    if missing:
        raise FileNotFoundError(f"reference sources not found: {missing}")
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    load(name="ctlab_ref_C", sources=src, build_directory=OUT, extra_cflags=["-O2"],
         extra_cuda_cflags=["-O2", "-gencode", "arch=compute_100,code=sm_100"], verbose=verbose, with_cuda=True)
    return built_path()


def load_ref():
    """The compiled reference module, or None when it has not been built."""
    path = built_path()
    if path is None:
        return None
    import torch  # noqa: F401  (the extension links against torch)
    spec = importlib.util.spec_from_file_location("ctlab_ref_C", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build(verbose="-q" not in sys.argv))
