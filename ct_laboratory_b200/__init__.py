"""ct_laboratory_b200 — the Siddon ray-driven projector A and its adjoint A^T
of ct_laboratory, rebuilt for NVIDIA B200 (sm_100a).

The compute runs in libctlab_b200.so (C ABI: include/ctlab_b200.h); this
package mirrors the reference's Python API on top of it:

  ct_laboratory_b200._C            the reference's 13 compiled entry points
  ct_laboratory_b200.tomography    modules, autograd Functions, function API,
                                   fan-beam / cone-beam / StaticCT geometry

As in the reference, the tomography names are also re-exported flat.
"""
from . import _native  # noqa: F401  (fails loudly if the library is missing)
from . import tomography  # noqa: F401
from .tomography import *  # noqa: F401,F403

__version__ = "0.1.0"
