"""Projectors: the reference's tomography area (ct_laboratory.tomography),
on the B200 kernels of libctlab_b200.so."""
from .standard_image_transform import *  # noqa: F401,F403
from .ct_projector_2d_cuda import *  # noqa: F401,F403
from .ct_projector_2d_torch import *  # noqa: F401,F403
from .ct_projector_2d_autograd import *  # noqa: F401,F403
from .ct_projector_2d_module import *  # noqa: F401,F403
from .ct_projector_3d_torch import *  # noqa: F401,F403
from .ct_projector_3d_cuda import *  # noqa: F401,F403
from .ct_projector_3d_autograd import *  # noqa: F401,F403
from .ct_projector_3d_module import *  # noqa: F401,F403
from .fanbeam_projector_2d import *  # noqa: F401,F403
from .conebeam_projector_3d import *  # noqa: F401,F403
from .staticct_projector_2d import *  # noqa: F401,F403
from .staticct_projector_3d import *  # noqa: F401,F403
from .gather import *  # noqa: F401,F403
from .fixed_adjoint import *  # noqa: F401,F403
from .ct_projector_3d_subsets import *  # noqa: F401,F403
from .ct_projector_3d_multirot import *  # noqa: F401,F403
