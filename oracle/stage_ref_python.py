"""Stage the reference's Python projector layers for the drop-in test (test
infrastructure only).

    python oracle/stage_ref_python.py      # needs the reference checkout

Copies the reference's ``ct_laboratory/tomography/*.py`` (its modules,
autograd Functions, function API and geometry classes, which reach the
compiled kernels through ``import ct_laboratory._C``) from the read-only
checkout ($CTLAB_REFERENCE, else the checkout beside this repository) into
``oracle/_ref/py/ct_laboratory/tomography/``, next to an empty package marker
written here.  oracle/_ref is git-ignored: nothing of the reference enters
the repository's history, and the staged copy travels to the GPU box with the
working tree, where tests/test_gpu_reference_python.py imports it with
``ct_laboratory._C`` bound to this package's ``_C`` (and, to compare, to the
reference's own compiled module).
"""
from __future__ import annotations

import glob
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "py")


def staged_path():
    """The directory to put on sys.path, or None when nothing is staged."""
    return OUT if os.path.exists(os.path.join(OUT, "ct_laboratory", "tomography", "__init__.py")) else None


def stage():
    try:
        from oracle.reference_path import reference_root
    except ImportError:  # run as a script from oracle/
        from reference_path import reference_root
    src = os.path.join(reference_root(required=True), "ct_laboratory", "tomography")
    dst = os.path.join(OUT, "ct_laboratory", "tomography")
    os.makedirs(dst, exist_ok=True)
    files = sorted(glob.glob(os.path.join(src, "*.py")))
    if not files:
        raise FileNotFoundError(f"no reference tomography modules under {src}")
    for f in files:
        shutil.copyfile(f, os.path.join(dst, os.path.basename(f)))
    with open(os.path.join(OUT, "ct_laboratory", "__init__.py"), "w") as fh:
        fh.write("# package marker for the staged reference tomography layers (oracle/stage_ref_python.py)\n")
    return dst


if __name__ == "__main__":
    print(stage(), file=sys.stdout)
