"""Where the reference checkout is, for the recipes that read it (test
infrastructure only: building oracle/_ref and generating golden fixtures).

$CTLAB_REFERENCE when set, else a checkout named ``reference`` beside this
repository's root directory; None when neither exists.  Nothing on the GPU
box or in the product reads the reference.
"""
from __future__ import annotations

import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root(required=False):
    cand = os.environ.get("CTLAB_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    if os.path.isdir(cand):
        return cand
    if required:
        raise FileNotFoundError("reference checkout not found: set CTLAB_REFERENCE to its directory")
    return None
